// FP64 cell-model kernels (the plain method), state initialisation and
// state gather/scatter.  The mixed-precision kernels live in ode_mixed.cu,
// which is compiled with the fast FP32 math.
#include "ode_common.cuh"
#include "model_torord_endo.cuh"

MB_NS_BEGIN

// ---- ToRORd-fkatp endo, forward Euler (FP64 in either tissue precision) ----
// Fixed step: num_steps Euler steps per loop step (default_solvers.c:37-53).
// Adaptive: one error-controlled pass to cur_time + adapt_span, with the
// cell's dt / time_new / previous_dt in sv64 rows NEQ..NEQ+2
// (default_solvers.c:55-175); a cell that does not reach the end time within
// the pass limit keeps its state and is counted in ctrl->ode_unfinished.
constexpr int TORE_MAX_PASSES = 200000;

template <int MINB, bool ADAPTIVE>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_torord_endo(mb_ode_dev o, mb_ctrl *ctrl, const double *__restrict__ vin, double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double y[mb_tore::NEQ];
    y[0] = src[g];
    act_track(o, ctrl, t, y[0]);
#pragma unroll
    for (int s = 1; s < mb_tore::NEQ; ++s) y[s] = o.sv64[s * ld + t];
    double *w = out64(o);
    const size_t wl = out_ld(o);
    if (!ADAPTIVE) {
        const double dt = o.dt;
        for (int step = 0; step < o.num_steps; ++step) {
            double d[mb_tore::NEQ];
            mb_tore::rhs(y, stim, d);
#pragma unroll
            for (int s = 0; s < mb_tore::NEQ; ++s) y[s] = dt * d[s] + y[s];
        }
    } else {
        double h = o.sv64[(size_t)mb_tore::NEQ * ld + t];
        double tn = o.sv64[(size_t)(mb_tore::NEQ + 1) * ld + t];
        double pdt = o.sv64[(size_t)(mb_tore::NEQ + 2) * ld + t];
        const double now = ctrl ? ctrl->cur_time : o.cur_time;
        const mb_tore::Adaptive p{o.min_dt, o.max_dt, o.abs_tol, o.rel_tol, TORE_MAX_PASSES};
        if (!mb_tore::adaptive_step(y, stim, now + o.adapt_span, p, h, tn, pdt) && ctrl)
            atomicAdd(&ctrl->ode_unfinished, 1u);
        w[(size_t)mb_tore::NEQ * wl + t] = h;
        w[(size_t)(mb_tore::NEQ + 1) * wl + t] = tn;
        w[(size_t)(mb_tore::NEQ + 2) * wl + t] = pdt;
    }
    vout[g] = y[0];
#pragma unroll
    for (int s = 1; s < mb_tore::NEQ; ++s) w[s * wl + t] = y[s];
}

// Row of state s in the (precision, model) layout: returns row and whether it
// is a double row.
__device__ __forceinline__ int state_row(int model, int precision, int s, bool &is64) {
    if (precision == MB_PREC_FP64) { is64 = true; return s; }
    if (model == MB_MODEL_TT2006) {
        switch (s) {
        case 0: is64 = true; return 0;
        case 13: is64 = true; return 1;
        case 14: is64 = true; return 2;
        case 15: is64 = true; return 3;
        case 17: is64 = true; return 4;
        case 18: is64 = true; return 5;
        case 16: is64 = false; return 12;
        default: is64 = false; return s - 1;   // gates 1..12 -> rows 0..11
        }
    }
    return tor_mixed_row(s, is64);
}

// Initial conditions from a table of ntypes x neq values, picked by celltype.
__global__ void k_ode_init(mb_ode_dev o, const double *__restrict__ table, int ntypes, int neq) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    int ct = 0;
    if (ntypes > 1 && o.celltype) ct = min((int)o.celltype[t], ntypes - 1);
    const double *ic = table + (size_t)ct * neq;
    for (int s = 0; s < neq; ++s) {
        bool is64;
        const int r = state_row(o.model, o.precision, s, is64);
        if (is64) o.sv64[(size_t)r * o.ld + t] = ic[s];
        else o.sv32[(size_t)r * o.ld + t] = (float)ic[s];
    }
}

// Dense copy of the state: out[s * n + t]; V comes from v[cell[t]] when v is
// given, else from row 0.
__global__ void k_ode_gather(mb_ode_dev o, const double *__restrict__ v, double *__restrict__ out, int neq) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    for (int s = 0; s < neq; ++s) {
        double val;
        if (s == 0 && v) {
            val = v[o.cell ? o.cell[t] : t];
        } else {
            bool is64;
            const int r = state_row(o.model, o.precision, s, is64);
            val = is64 ? o.sv64[(size_t)r * o.ld + t] : (double)o.sv32[(size_t)r * o.ld + t];
        }
        out[(size_t)s * o.n + t] = val;
    }
}

__global__ void k_ode_scatter(mb_ode_dev o, const double *__restrict__ in, double *__restrict__ v, int neq) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    for (int s = 0; s < neq; ++s) {
        const double val = in[(size_t)s * o.n + t];
        if (s == 0 && v) { v[o.cell ? o.cell[t] : t] = val; continue; }
        bool is64;
        const int r = state_row(o.model, o.precision, s, is64);
        if (is64) o.sv64[(size_t)r * o.ld + t] = val;
        else o.sv32[(size_t)r * o.ld + t] = (float)val;
    }
}

MB_NS_END

using namespace mb;

static int neq_of(int model) { return model == MB_MODEL_TT2006 ? TT_NEQ : TOR_NEQ; }

extern "C" int mbk_ode_init(const mb_ode_dev *o, const double *table_dev, int ntypes, cudaStream_t s) {
    if (o->n == 0) return 0;
    k_ode_init<<<(o->n + 127) / 128, 128, 0, s>>>(*o, table_dev, ntypes, neq_of(o->model));
    return (int)cudaGetLastError();
}

extern "C" int mbk_ode_step(const mb_ode_dev *o, mb_ctrl *ctrl, const double *vin, double *vout, cudaStream_t s) {
    if (o->n == 0) return 0;
    const unsigned blocks = (o->n + ODE_THREADS - 1) / ODE_THREADS;
    const mb_ode_dev &a = *o;
    if (o->model == MB_MODEL_TORORD_FKATP_ENDO) {
        // one-launch kernels only (the staged variants fall back to them)
#define L(MB, AD) k_torord_endo<MB, AD><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
        if (o->adaptive) {
            L(1, true);
        } else {
            switch (o->variant) {
            case 0: L(1, false); break;
            case 1: L(2, false); break;
            case 2: L(3, false); break;
            default: L(4, false); break;
            }
        }
#undef L
        return (int)cudaGetLastError();
    }
    if (o->precision != MB_PREC_FP64) return mbk_ode_step_mixed(o, ctrl, vin, vout, s);
#define MB_STAGED(KERNEL, N64, N32)                                                       \
    do {                                                                                  \
        const size_t sm = staged_smem(N64, N32);                                          \
        auto *kfn = KERNEL;                                                               \
        const unsigned gb = staged_grid((const void *)kfn, sm, blocks);                   \
        if (!gb) return (int)cudaErrorInvalidConfiguration;                               \
        kfn<<<gb, ODE_THREADS, sm, s>>>(a, ctrl, vin, vout);                              \
    } while (0)
    if (o->model == MB_MODEL_TT2006) {
#define L(MB) k_tt2006_fp64<MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
#define LS(MB) MB_STAGED(k_tt2006_fp64_s<MB>, TT_NEQ, 0)
        MB_VARIANT_SWITCH(o->variant, L, LS)
#undef L
#undef LS
    } else if (o->rl_rule == MB_RL_TRUE) {
#define L(MB) k_torord_fp64<MB_RL_TRUE, MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
#define LS(MB) MB_STAGED((k_torord_fp64_s<MB_RL_TRUE, MB>), TOR_NEQ, 0)
        MB_VARIANT_SWITCH(o->variant, L, LS)
#undef L
#undef LS
    } else {
#define L(MB) k_torord_fp64<MB_RL_REFERENCE_CPU, MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
#define LS(MB) MB_STAGED((k_torord_fp64_s<MB_RL_REFERENCE_CPU, MB>), TOR_NEQ, 0)
        MB_VARIANT_SWITCH(o->variant, L, LS)
#undef L
#undef LS
    }
#undef MB_STAGED
    return (int)cudaGetLastError();
}

extern "C" int mbk_ode_gather(const mb_ode_dev *o, const double *v, double *out_dev, cudaStream_t s) {
    if (o->n == 0) return 0;
    k_ode_gather<<<(o->n + 127) / 128, 128, 0, s>>>(*o, v, out_dev, neq_of(o->model));
    return (int)cudaGetLastError();
}

extern "C" int mbk_ode_scatter(const mb_ode_dev *o, const double *in_dev, double *v, cudaStream_t s) {
    if (o->n == 0) return 0;
    k_ode_scatter<<<(o->n + 127) / 128, 128, 0, s>>>(*o, in_dev, v, neq_of(o->model));
    return (int)cudaGetLastError();
}

extern "C" double mb_tt2006_default_state(int s) { return tt2006_default_state(s); }
extern "C" double mb_torord_default_state(int celltype, int s) { return torord_default_state(celltype, s); }
extern "C" double mb_torord_endo_default_state(int gpu_build, int s) {
    return gpu_build ? mb_tore::initial_state_gpu(s) : mb_tore::initial_state_cpu(s);
}

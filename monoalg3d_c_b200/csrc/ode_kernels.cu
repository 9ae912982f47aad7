// FP64 cell-model kernels (the plain method), state initialisation and
// state gather/scatter.  The mixed-precision kernels live in ode_mixed.cu,
// which is compiled with the fast FP32 math.
#include "ode_common.cuh"

MB_NS_BEGIN

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
    if (o->precision != MB_PREC_FP64) return mbk_ode_step_mixed(o, ctrl, vin, vout, s);
    const unsigned blocks = (o->n + ODE_THREADS - 1) / ODE_THREADS;
    const mb_ode_dev &a = *o;
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

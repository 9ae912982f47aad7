// Per-cell ionic ODE kernels: one thread per cell, state in structure-of-arrays
// rows so that every row load/store of a warp is one coalesced 128/256-byte
// transaction; all num_steps sub-steps run with the state in registers.
//
// Reference behaviour followed:
//   sub-step loop per cell        ten_tusscher_2006_RS_CPU.c:74-98,
//                                 ToRORd_fkatp_mixed_endo_mid_epi.c:165-250
//   stimulus merge per sub-step   ode_solver.c:201-235 (window inclusive)
//   V taken from the grid only when cur_time > 0
//                                 monodomain_solver.c:660-661
#include <cstdint>
#include "mb_internal.h"
#include "model_tt2006.cuh"
#include "model_torord.cuh"

namespace mb {

// Merged stimulus of compact cell t for the current loop step: every stimulus
// config whose bit is set adds its current once per sub-step whose time lies
// in [start, start + duration] (ode_solver.c:213-222).
__device__ __forceinline__ double cell_stim(const mb_ode_dev &o, const mb_ctrl *__restrict__ c,
                                            uint32_t t) {
    if (o.stim_host) return o.stim_host[t];
    if (!o.stim_bits) return 0.0;
    const unsigned bits = o.stim_bits[t];
    if (!bits) return 0.0;
    double s = 0.0;
    const int ns = c->num_stims;
    for (int k = 0; k < ns; ++k) {
        if (!((bits >> k) & 1u)) continue;
        const double start = c->stim_start[k];
        const double end = start + c->stim_dur[k];
        const double cur = c->stim_current[k];
        double time = c->cur_time;
        for (int j = 0; j < o.num_steps; ++j) {
            if (time >= start && time <= end) s += cur;
            time += o.dt;
        }
    }
    return s;
}

template <typename T>
__device__ __forceinline__ TTScale<T> load_tt_scale(const mb_ode_dev &o, uint32_t t) {
    TTScale<T> sc;
    if (o.scale) {
        sc.gNa = T(o.scale[0 * (size_t)o.ld + t]);
        sc.gKr = T(o.scale[1 * (size_t)o.ld + t]);
        sc.gKs = T(o.scale[2 * (size_t)o.ld + t]);
        sc.gCaL = T(o.scale[3 * (size_t)o.ld + t]);
        sc.gK1 = T(o.scale[4 * (size_t)o.ld + t]);
    } else {
        sc.gNa = sc.gKr = sc.gKs = sc.gCaL = sc.gK1 = T(1);
    }
    return sc;
}

// ---- ten Tusscher 2006 --------------------------------------------------
// FP64 layout: sv64 row s = state s (row 0 unused when V lives in the grid).
// Mixed layout: sv64 rows {V, Ca_i, Ca_SR, Ca_ss, Na_i, K_i};
//               sv32 rows {Xr1 .. r (12 gates), R'}.
__global__ void __launch_bounds__(128) k_tt2006_fp64(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl,
                                                     const double *__restrict__ vin,
                                                     double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double y[TT_NEQ];
    y[0] = src[g];
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) y[s] = o.sv64[s * ld + t];
    const TTScale<double> sc = load_tt_scale<double>(o, t);
    const double dt = o.dt;
    for (int step = 0; step < o.num_steps; ++step) {
        TTUpdate<double> u;
        tt2006_rhs<double>(y, stim, dt, sc, u);
        y[TT_V] = dt * u.dV + y[TT_V];
#pragma unroll
        for (int k = 0; k < 12; ++k) y[1 + k] = u.gate[k];
        y[TT_CAI] = dt * u.dCai + y[TT_CAI];
        y[TT_CASR] = dt * u.dCaSR + y[TT_CASR];
        y[TT_CASS] = dt * u.dCaSS + y[TT_CASS];
        y[TT_RPRIME] = dt * u.dRprime + y[TT_RPRIME];
        y[TT_NAI] = dt * u.dNai + y[TT_NAI];
        y[TT_KI] = dt * u.dKi + y[TT_KI];
    }
    vout[g] = y[0];
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) o.sv64[s * ld + t] = y[s];
}

__global__ void __launch_bounds__(128) k_tt2006_mixed(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl,
                                                      const double *__restrict__ vin,
                                                      double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const float stim = (float)cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double V = src[g];
    double cai = o.sv64[1 * ld + t], casr = o.sv64[2 * ld + t], cass = o.sv64[3 * ld + t];
    double nai = o.sv64[4 * ld + t], ki = o.sv64[5 * ld + t];
    float gates[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) gates[k] = o.sv32[k * ld + t];
    float rprime = o.sv32[12 * ld + t];
    const TTScale<float> sc = load_tt_scale<float>(o, t);
    const double dt = o.dt;
    const float dtf = (float)dt;
    for (int step = 0; step < o.num_steps; ++step) {
        float y[TT_NEQ];
        y[TT_V] = (float)V;
#pragma unroll
        for (int k = 0; k < 12; ++k) y[1 + k] = gates[k];
        y[TT_CAI] = (float)cai; y[TT_CASR] = (float)casr; y[TT_CASS] = (float)cass;
        y[TT_RPRIME] = rprime; y[TT_NAI] = (float)nai; y[TT_KI] = (float)ki;
        TTUpdate<float> u;
        tt2006_rhs<float>(y, stim, dtf, sc, u);
        V = dt * (double)u.dV + V;
#pragma unroll
        for (int k = 0; k < 12; ++k) gates[k] = u.gate[k];
        cai = dt * (double)u.dCai + cai;
        casr = dt * (double)u.dCaSR + casr;
        cass = dt * (double)u.dCaSS + cass;
        rprime = dtf * u.dRprime + rprime;
        nai = dt * (double)u.dNai + nai;
        ki = dt * (double)u.dKi + ki;
    }
    vout[g] = V;
    o.sv64[1 * ld + t] = cai; o.sv64[2 * ld + t] = casr; o.sv64[3 * ld + t] = cass;
    o.sv64[4 * ld + t] = nai; o.sv64[5 * ld + t] = ki;
#pragma unroll
    for (int k = 0; k < 12; ++k) o.sv32[k * ld + t] = gates[k];
    o.sv32[12 * ld + t] = rprime;
}

// ---- ToRORd-fkatp endo/mid/epi -------------------------------------------
// FP64 layout: sv64 row s = state s.
// Mixed layout: sv64 rows = TOR_ROWS64 (V and the 8 ion concentrations),
//               sv32 rows = the other 34 states in index order.
template <int RULE>
__global__ void __launch_bounds__(128) k_torord_fp64(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl,
                                                     const double *__restrict__ vin,
                                                     double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double y[TOR_NEQ];
    y[0] = src[g];
#pragma unroll
    for (int s = 1; s < TOR_NEQ; ++s) y[s] = o.sv64[s * ld + t];
    const double celltype = o.celltype ? (double)o.celltype[t] : 0.0;
    TorScale<double> sc;
    load_tor_scale(o.scale, ld, t, sc);
    const double dt = o.dt;
    for (int step = 0; step < o.num_steps; ++step) torord_rl_step<double, double, RULE>(y, stim, dt, celltype, sc);
    vout[g] = y[0];
#pragma unroll
    for (int s = 1; s < TOR_NEQ; ++s) o.sv64[s * ld + t] = y[s];
}

template <int RULE>
__global__ void __launch_bounds__(128) k_torord_mixed(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl,
                                                      const double *__restrict__ vin,
                                                      double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    TorMixedState st;
    st.d[0] = src[g];
#pragma unroll
    for (int r = 1; r < TOR_N64; ++r) st.d[r] = o.sv64[r * ld + t];
#pragma unroll
    for (int r = 0; r < TOR_N32; ++r) st.f[r] = o.sv32[r * ld + t];
    const float celltype = o.celltype ? (float)o.celltype[t] : 0.0f;
    TorScale<float> sc;
    load_tor_scale(o.scale, ld, t, sc);
    const double dt = o.dt;
    for (int step = 0; step < o.num_steps; ++step) torord_mixed_step<RULE>(st, stim, dt, celltype, sc);
    vout[g] = st.d[0];
#pragma unroll
    for (int r = 1; r < TOR_N64; ++r) o.sv64[r * ld + t] = st.d[r];
#pragma unroll
    for (int r = 0; r < TOR_N32; ++r) o.sv32[r * ld + t] = st.f[r];
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

}  // namespace mb

using namespace mb;

static int neq_of(int model) { return model == MB_MODEL_TT2006 ? TT_NEQ : TOR_NEQ; }

extern "C" int mbk_ode_init(const mb_ode_dev *o, const double *table_dev, int ntypes, cudaStream_t s) {
    if (o->n == 0) return 0;
    const unsigned blocks = (o->n + 127) / 128;
    k_ode_init<<<blocks, 128, 0, s>>>(*o, table_dev, ntypes, neq_of(o->model));
    return (int)cudaGetLastError();
}

extern "C" int mbk_ode_step(const mb_ode_dev *o, mb_ctrl *ctrl, const double *vin, double *vout,
                            cudaStream_t s) {
    if (o->n == 0) return 0;
    const unsigned blocks = (o->n + 127) / 128;
    if (o->model == MB_MODEL_TT2006) {
        if (o->precision == MB_PREC_FP64) k_tt2006_fp64<<<blocks, 128, 0, s>>>(*o, ctrl, vin, vout);
        else k_tt2006_mixed<<<blocks, 128, 0, s>>>(*o, ctrl, vin, vout);
    } else {
        if (o->precision == MB_PREC_FP64) {
            if (o->rl_rule == MB_RL_TRUE) k_torord_fp64<MB_RL_TRUE><<<blocks, 128, 0, s>>>(*o, ctrl, vin, vout);
            else k_torord_fp64<MB_RL_REFERENCE_CPU><<<blocks, 128, 0, s>>>(*o, ctrl, vin, vout);
        } else {
            if (o->rl_rule == MB_RL_TRUE) k_torord_mixed<MB_RL_TRUE><<<blocks, 128, 0, s>>>(*o, ctrl, vin, vout);
            else k_torord_mixed<MB_RL_REFERENCE_CPU><<<blocks, 128, 0, s>>>(*o, ctrl, vin, vout);
        }
    }
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

extern "C" double mb_tt2006_default_state(int s) { return mb::tt2006_default_state(s); }
extern "C" double mb_torord_default_state(int celltype, int s) { return mb::torord_default_state(celltype, s); }

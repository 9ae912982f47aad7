// Per-cell ionic ODE kernels: one thread per cell, state in structure-of-arrays
// rows so that every row load/store of a warp is one coalesced transaction;
// all num_steps sub-steps run with the state in registers.  MINB is the
// minimum number of resident 128-thread blocks per SM the register allocation
// must allow (the autotuner picks one per model and precision).
//
// Reference behaviour followed:
//   sub-step loop per cell        ten_tusscher_2006_RS_CPU.c:74-98,
//                                 ToRORd_fkatp_mixed_endo_mid_epi.c:165-250
//   stimulus merge per sub-step   ode_solver.c:201-235 (window inclusive)
//   V taken from the grid only when cur_time > 0
//                                 monodomain_solver.c:660-661
#pragma once
#include <cstdint>
#include "mb_internal.h"
#include "model_tt2006.cuh"
#include "model_torord.cuh"

MB_NS_BEGIN

constexpr int ODE_THREADS = 128;

// Merged stimulus of compact cell t for the current loop step: every stimulus
// config whose bit is set adds its current once per sub-step whose time lies
// in [start, start + duration] (ode_solver.c:213-222).
__device__ __forceinline__ double cell_stim(const mb_ode_dev &o, const mb_ctrl *__restrict__ c, uint32_t t) {
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

// Activation time and APD90 of compact cell t from V at the start of the loop
// step (time cur_time).  An activation is an upward crossing of
// act_threshold (the reference's activation_threshold, save_mesh.c:787-848)
// at least act_min_interval after the previous one (its time_threshold), its
// time linearly interpolated between the two loop steps.  APD90 ends at the
// downward crossing, after the peak, of V_peak - 0.9 (V_peak - V_rest) with
// V_rest the lowest V since the previous repolarisation, also interpolated.
__device__ __forceinline__ void act_track(const mb_ode_dev &o, const mb_ctrl *__restrict__ c, uint32_t t,
                                          double Vd) {
    if (o.act == nullptr || c == nullptr) return;
    float *a = o.act;
    const size_t ld = o.ld;
    const float V = (float)Vd;
    const float vp = a[MB_ACT_VPREV * ld + t];
    if (isnan(vp)) {
        a[MB_ACT_VPREV * ld + t] = V;
        a[MB_ACT_VREST * ld + t] = V;
        return;
    }
    const double tc = c->cur_time, dt = c->act_dt;
    int state = (int)a[MB_ACT_STATE * ld + t];
    int n = state >> 1, phase = state & 1;
    const float thr = c->act_threshold;
    if (vp < thr && V >= thr) {
        const float tl = a[MB_ACT_LAST * ld + t];
        if (tl < 0.0f || tc - (double)tl > (double)c->act_min_interval) {
            const float ta = (float)((tc - dt) + dt * (double)(thr - vp) / (double)(V - vp));
            if (n == 0) a[MB_ACT_FIRST * ld + t] = ta;
            a[MB_ACT_LAST * ld + t] = ta;
            a[MB_ACT_APD * ld + t] = -1.0f;
            a[MB_ACT_VPEAK * ld + t] = V;
            n += 1;
            phase = 1;
        }
    }
    if (phase) {
        const float pk = fmaxf(a[MB_ACT_VPEAK * ld + t], V);
        a[MB_ACT_VPEAK * ld + t] = pk;
        const float rest = a[MB_ACT_VREST * ld + t];
        const float v90 = pk - 0.9f * (pk - rest);
        if (vp > v90 && V <= v90 && V < pk) {
            const double tr = (tc - dt) + dt * (double)(vp - v90) / (double)(vp - V);
            a[MB_ACT_APD * ld + t] = (float)(tr - (double)a[MB_ACT_LAST * ld + t]);
            a[MB_ACT_VREST * ld + t] = V;
            phase = 0;
        }
    } else {
        const float rest = a[MB_ACT_VREST * ld + t];
        if (V < rest) a[MB_ACT_VREST * ld + t] = V;
    }
    a[MB_ACT_VPREV * ld + t] = V;
    a[MB_ACT_STATE * ld + t] = (float)(2 * n + phase);
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

// Where the new state goes: in place, or into the tuning buffers.
__device__ __forceinline__ double *out64(const mb_ode_dev &o) { return o.out64 ? o.out64 : o.sv64; }
__device__ __forceinline__ float *out32(const mb_ode_dev &o) { return o.out64 ? o.out32 : o.sv32; }
__device__ __forceinline__ size_t out_ld(const mb_ode_dev &o) { return o.out64 ? o.out_ld : o.ld; }

// ---- ten Tusscher 2006 ----------------------------------------------------
// FP64 layout: sv64 row s = state s (row 0 unused when V lives in the grid).
// Mixed layout: sv64 rows {V, Ca_i, Ca_SR, Ca_ss, Na_i, K_i};
//               sv32 rows {Xr1 .. r (12 gates), R'}.
template <int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_tt2006_fp64(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
              double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double y[TT_NEQ];
    y[0] = src[g];
    act_track(o, ctrl, t, y[0]);
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
    double *w = out64(o);
    const size_t wl = out_ld(o);
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) w[s * wl + t] = y[s];
}

template <int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_tt2006_mixed(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
               double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const float stim = (float)cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double V = src[g];
    act_track(o, ctrl, t, V);
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
    double *w = out64(o);
    float *w32 = out32(o);
    const size_t wl = out_ld(o);
    w[1 * wl + t] = cai; w[2 * wl + t] = casr; w[3 * wl + t] = cass;
    w[4 * wl + t] = nai; w[5 * wl + t] = ki;
#pragma unroll
    for (int k = 0; k < 12; ++k) w32[k * wl + t] = gates[k];
    w32[12 * wl + t] = rprime;
}

// ---- ToRORd-fkatp endo/mid/epi -------------------------------------------
// FP64 layout: sv64 row s = state s.
// Mixed layout: sv64 rows {V, cass, nai, nass, ki, kss, cansr, cajsr, cai},
//               sv32 rows {CaMKt, states 10..42}.
template <int RULE, int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_torord_fp64(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
              double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    double y[TOR_NEQ];
    y[0] = src[g];
    act_track(o, ctrl, t, y[0]);
#pragma unroll
    for (int s = 1; s < TOR_NEQ; ++s) y[s] = o.sv64[s * ld + t];
    const double celltype = o.celltype ? (double)o.celltype[t] : 0.0;
    TorScale<double> sc;
    load_tor_scale(o.scale, ld, t, sc);
    const double dt = o.dt;
    for (int step = 0; step < o.num_steps; ++step) torord_rl_step<double, double, RULE>(y, stim, dt, celltype, sc);
    vout[g] = y[0];
    double *w = out64(o);
    const size_t wl = out_ld(o);
#pragma unroll
    for (int s = 1; s < TOR_NEQ; ++s) w[s * wl + t] = y[s];
}

template <int RULE, int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_torord_mixed(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
               double *__restrict__ vout) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const double stim = cell_stim(o, ctrl, t);
    const size_t ld = o.ld;
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    TorMixedState st;
    st.d[0] = src[g];
    act_track(o, ctrl, t, st.d[0]);
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
    double *w = out64(o);
    float *w32 = out32(o);
    const size_t wl = out_ld(o);
#pragma unroll
    for (int r = 1; r < TOR_N64; ++r) w[r * wl + t] = st.d[r];
#pragma unroll
    for (int r = 0; r < TOR_N32; ++r) w32[r * wl + t] = st.f[r];
}

// ---- staged persistent form ----------------------------------------------
// The same per-cell work in a persistent loop over tiles of ODE_THREADS
// cells.  While a thread integrates its cell of one tile, the state rows of
// its cell in the next tile are being copied into its own slots of shared
// memory (cp.async), and that cell's grid index, stimulus bits / external
// stimulus and cell type are loaded into registers, so the latency of the
// state loads overlaps the integration instead of stalling it.  A thread
// reads only the shared-memory slots it filled itself, so no barrier is
// needed; the copies of a tile are waited for with cp.async.wait_group.

__device__ __forceinline__ void cpa4(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa8(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared memory of a staged block: two tiles of N64 double rows (row 0 = V)
// and N32 float rows.
__host__ __device__ constexpr size_t staged_smem(int n64, int n32) {
    return 2 * (size_t)ODE_THREADS * ((size_t)n64 * 8 + (size_t)n32 * 4);
}

// Per-cell values loaded a tile ahead.
struct CellAhead {
    uint32_t g;      // grid index (V)
    uint32_t bits;   // stimulus bits | cell type << 8
    double sh;       // external stimulus (reference-host mode)
};

__device__ __forceinline__ CellAhead cell_ahead(const mb_ode_dev &o, uint32_t t) {
    CellAhead e{0u, 0u, 0.0};
    if (t < o.n) {
        e.g = o.cell ? o.cell[t] : t;
        if (o.stim_host) e.sh = o.stim_host[t];
        else if (o.stim_bits) e.bits = o.stim_bits[t];
        if (o.celltype) e.bits |= (uint32_t)o.celltype[t] << 8;
    }
    return e;
}

// cell_stim from the prefetched bits (the same sum, ode_solver.c:213-222)
__device__ __forceinline__ double stim_ahead(const mb_ode_dev &o, const mb_ctrl *__restrict__ c, const CellAhead &e) {
    if (o.stim_host) return e.sh;
    const unsigned bits = e.bits & 0xffu;
    if (!o.stim_bits || !bits) return 0.0;
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

// The persistent tile loop: work(t, ahead, d, f) integrates cell t from its
// state d (N64 doubles, d[0] = V) and f (N32 floats) and stores the results.
template <int N64, int N32, typename W>
__device__ __forceinline__ void staged_cells(const mb_ode_dev &o, const double *__restrict__ src, W work) {
    extern __shared__ __align__(16) unsigned char ode_smem[];
    double *b64 = reinterpret_cast<double *>(ode_smem);
    float *b32 = reinterpret_cast<float *>(ode_smem + (size_t)2 * N64 * ODE_THREADS * 8);
    const uint32_t tid = threadIdx.x, T = ODE_THREADS;
    const uint32_t ntiles = (o.n + T - 1) / T;
    const size_t ld = o.ld;
    auto stage = [&](uint32_t tile, uint32_t g, int b) {
        const uint32_t t = tile * T + tid;
        if (tile < ntiles && t < o.n) {
            cpa8(&b64[(size_t)(b * N64) * T + tid], src + g);
#pragma unroll
            for (int r = 1; r < N64; ++r) cpa8(&b64[(size_t)(b * N64 + r) * T + tid], o.sv64 + r * ld + t);
#pragma unroll
            for (int r = 0; r < N32; ++r) cpa4(&b32[(size_t)(b * N32 + r) * T + tid], o.sv32 + r * ld + t);
        }
        cpa_commit();
    };
    uint32_t tile = blockIdx.x;
    CellAhead cur = cell_ahead(o, tile * T + tid);
    stage(tile, cur.g, 0);
    CellAhead nxt = cell_ahead(o, (tile + gridDim.x) * T + tid);
    int b = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        const uint32_t tn = tile + gridDim.x;
        stage(tn, nxt.g, b ^ 1);
        const CellAhead after = cell_ahead(o, (tn + gridDim.x) * T + tid);
        cpa_wait1();
        const uint32_t t = tile * T + tid;
        if (t < o.n) {
            double d[N64];
            float f[N32 > 0 ? N32 : 1];
#pragma unroll
            for (int r = 0; r < N64; ++r) d[r] = b64[(size_t)(b * N64 + r) * T + tid];
#pragma unroll
            for (int r = 0; r < N32; ++r) f[r] = b32[(size_t)(b * N32 + r) * T + tid];
            work(t, cur, d, f);
        }
        cur = nxt;
        nxt = after;
        b ^= 1;
    }
    cpa_wait0();
}

template <int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_tt2006_fp64_s(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
                double *__restrict__ vout) {
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    staged_cells<TT_NEQ, 0>(o, src, [&](uint32_t t, const CellAhead &e, double (&y)[TT_NEQ], float (&)[1]) {
        act_track(o, ctrl, t, y[0]);
        const double stim = stim_ahead(o, ctrl, e);
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
        vout[e.g] = y[0];
        double *w = out64(o);
        const size_t wl = out_ld(o);
#pragma unroll
        for (int s = 1; s < TT_NEQ; ++s) w[s * wl + t] = y[s];
    });
}

template <int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_tt2006_mixed_s(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
                 double *__restrict__ vout) {
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    // staged rows: V, sv64 rows 1..5 (Ca_i, Ca_SR, Ca_ss, Na_i, K_i); sv32 rows 0..12
    staged_cells<6, 13>(o, src, [&](uint32_t t, const CellAhead &e, double (&d)[6], float (&f)[13]) {
        double V = d[0];
        act_track(o, ctrl, t, V);
        double cai = d[1], casr = d[2], cass = d[3], nai = d[4], ki = d[5];
        float gates[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) gates[k] = f[k];
        float rprime = f[12];
        const float stim = (float)stim_ahead(o, ctrl, e);
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
        vout[e.g] = V;
        double *w = out64(o);
        float *w32 = out32(o);
        const size_t wl = out_ld(o);
        w[1 * wl + t] = cai; w[2 * wl + t] = casr; w[3 * wl + t] = cass;
        w[4 * wl + t] = nai; w[5 * wl + t] = ki;
#pragma unroll
        for (int k = 0; k < 12; ++k) w32[k * wl + t] = gates[k];
        w32[12 * wl + t] = rprime;
    });
}

template <int RULE, int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_torord_fp64_s(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
                double *__restrict__ vout) {
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    staged_cells<TOR_NEQ, 0>(o, src, [&](uint32_t t, const CellAhead &e, double (&y)[TOR_NEQ], float (&)[1]) {
        act_track(o, ctrl, t, y[0]);
        const double stim = stim_ahead(o, ctrl, e);
        const double celltype = (double)(e.bits >> 8);
        TorScale<double> sc;
        load_tor_scale(o.scale, o.ld, t, sc);
        const double dt = o.dt;
        for (int step = 0; step < o.num_steps; ++step) torord_rl_step<double, double, RULE>(y, stim, dt, celltype, sc);
        vout[e.g] = y[0];
        double *w = out64(o);
        const size_t wl = out_ld(o);
#pragma unroll
        for (int s = 1; s < TOR_NEQ; ++s) w[s * wl + t] = y[s];
    });
}

template <int RULE, int MINB>
__global__ void __launch_bounds__(ODE_THREADS, MINB)
k_torord_mixed_s(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl, const double *__restrict__ vin,
                 double *__restrict__ vout) {
    const double *src = (ctrl == nullptr || ctrl->cur_time > 0.0) ? vin : vout;
    staged_cells<TOR_N64, TOR_N32>(o, src, [&](uint32_t t, const CellAhead &e, double (&d)[TOR_N64],
                                                float (&f)[TOR_N32]) {
        TorMixedState st;
#pragma unroll
        for (int r = 0; r < TOR_N64; ++r) st.d[r] = d[r];
#pragma unroll
        for (int r = 0; r < TOR_N32; ++r) st.f[r] = f[r];
        act_track(o, ctrl, t, st.d[0]);
        const double stim = stim_ahead(o, ctrl, e);
        const float celltype = (float)(e.bits >> 8);
        TorScale<float> sc;
        load_tor_scale(o.scale, o.ld, t, sc);
        const double dt = o.dt;
        for (int step = 0; step < o.num_steps; ++step) torord_mixed_step<RULE>(st, stim, dt, celltype, sc);
        vout[e.g] = st.d[0];
        double *w = out64(o);
        float *w32 = out32(o);
        const size_t wl = out_ld(o);
#pragma unroll
        for (int r = 1; r < TOR_N64; ++r) w[r * wl + t] = st.d[r];
#pragma unroll
        for (int r = 0; r < TOR_N32; ++r) w32[r * wl + t] = st.f[r];
    });
}

// Grid of a staged kernel: every SM filled to the occupancy its registers
// and shared memory allow (the kernel loops over the tiles).
inline unsigned staged_grid(const void *fn, size_t smem, unsigned tiles) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, ODE_THREADS, smem) != cudaSuccess || per < 1)
        return 0;
    const unsigned g = (unsigned)(sms * per);
    return g < tiles ? g : tiles;
}

// Launch of one (model, precision) family: variants 0..5 are the one-cell-
// per-thread kernels with at least 1..6 resident blocks per SM, 6..9 the
// staged kernels with at least 1..4.  A staged launch that cannot be placed
// (shared memory) returns cudaErrorInvalidConfiguration.
#define MB_VARIANT_SWITCH(variant, LAUNCH, LAUNCH_S) \
    switch (variant) {                               \
    case 0: LAUNCH(1); break;                        \
    case 1: LAUNCH(2); break;                        \
    case 2: LAUNCH(3); break;                        \
    case 3: LAUNCH(4); break;                        \
    case 4: LAUNCH(5); break;                        \
    case 5: LAUNCH(6); break;                        \
    case 6: LAUNCH_S(1); break;                      \
    case 7: LAUNCH_S(2); break;                      \
    case 8: LAUNCH_S(3); break;                      \
    default: LAUNCH_S(4); break;                     \
    }

MB_NS_END

// Kernels of the discrete adjoint of the monodomain step (ten Tusscher 2006,
// per-cell conductivity, FP64).
//
// One loop step maps (v_n, s_n) to v_{n+1} through
//     (V*, s_{n+1}) = Phi(v_n, s_n; theta)       Rush-Larsen sub-step
//     A(sigma) v_{n+1} = alpha V*                implicit diffusion
// and its adjoint, run backwards, maps (lambda_{n+1} = dL/dv_{n+1},
// mu_{n+1} = dL/ds_{n+1}) to (lambda_n, mu_n):
//     A w = lambda_{n+1}                          (A is symmetric: the same PCG)
//     dL/dsigma += -(w_a - w_b)(v_a - v_b) dF_ab/dsigma  over faces ab
//     (lambda_n, mu_n, dL/dtheta) = J_Phi^T (alpha w, mu_{n+1})
// J_Phi^T is formed column block by column block with forward-mode dual
// numbers through the same templated model code the forward kernels run
// (model_tt2006.cuh), so the adjoint differentiates exactly the arithmetic of
// the forward step.
#include <cstdint>
#include <cuda_runtime.h>
#include "mb_internal.h"
#include "ode_common.cuh"

MB_NS_BEGIN

// ---- dual numbers ---------------------------------------------------------------

// value type T: double for the FP64 forward, float for the mixed one
template <int K, typename T = double>
struct Dual {
    T v;
    T d[K];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v((T)x) {
#pragma unroll
        for (int k = 0; k < K; ++k) d[k] = T(0);
    }
};

#define MB_DUAL_BIN(OP, VAL, DER)                                                                      \
    template <int K, typename T>                                                                       \
    __device__ __forceinline__ Dual<K, T> operator OP(const Dual<K, T> &a, const Dual<K, T> &b) {      \
        Dual<K, T> r;                                                                                  \
        r.v = VAL;                                                                                     \
        _Pragma("unroll") for (int k = 0; k < K; ++k) r.d[k] = DER;                                    \
        return r;                                                                                      \
    }
MB_DUAL_BIN(+, a.v + b.v, a.d[k] + b.d[k])
MB_DUAL_BIN(-, a.v - b.v, a.d[k] - b.d[k])
MB_DUAL_BIN(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
MB_DUAL_BIN(/, a.v / b.v, (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v))
#undef MB_DUAL_BIN

template <int K, typename T>
__device__ __forceinline__ Dual<K, T> operator-(const Dual<K, T> &a) {
    Dual<K, T> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int K, typename T>
__device__ __forceinline__ bool operator<(const Dual<K, T> &a, const Dual<K, T> &b) { return a.v < b.v; }
template <int K, typename T>
__device__ __forceinline__ bool operator>(const Dual<K, T> &a, const Dual<K, T> &b) { return a.v > b.v; }
template <int K, typename T>
__device__ __forceinline__ bool operator<=(const Dual<K, T> &a, const Dual<K, T> &b) { return a.v <= b.v; }
template <int K, typename T>
__device__ __forceinline__ bool operator>=(const Dual<K, T> &a, const Dual<K, T> &b) { return a.v >= b.v; }

template <int K, typename T>
__device__ __forceinline__ Dual<K, T> chain(const Dual<K, T> &a, T val, T der) {
    Dual<K, T> r;
    r.v = val;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = der * a.d[k];
    return r;
}
// the value-type functions mexp / mexpm1 / mlog / msqrt of mb_math.cuh
template <int K, typename T> __device__ __forceinline__ Dual<K, T> mexp(const Dual<K, T> &a) {
    const T e = mexp(a.v);
    return chain(a, e, e);
}
template <int K, typename T> __device__ __forceinline__ Dual<K, T> mexpm1(const Dual<K, T> &a) {
    return chain(a, mexpm1(a.v), mexp(a.v));
}
template <int K, typename T> __device__ __forceinline__ Dual<K, T> mlog(const Dual<K, T> &a) {
    return chain(a, mlog(a.v), T(1) / a.v);
}
template <int K, typename T> __device__ __forceinline__ Dual<K, T> msqrt(const Dual<K, T> &a) {
    const T s = msqrt(a.v);
    return chain(a, s, T(0.5) / s);
}

// ---- ODE adjoint ----------------------------------------------------------------

constexpr int ADJ_THREADS = 128;
constexpr int ADJ_IN = TT_NEQ + 1;      // the 19 states and the gKr scaling

// Column block [j0, j0 + K) of J_Phi, contracted with g: res[j] += sum_i g_i
// d(out_i)/d(in_j).  Inputs 0..18 are the states (0 = V), input 19 the gKr
// scaling.  T: the arithmetic of the forward step (double; float for the
// mixed form, whose right-hand side is FP32); the contraction with g and the
// results are FP64.
template <int K, typename T = double>
__device__ __forceinline__ void adj_block(int j0, const T (&y)[TT_NEQ], const TTScale<T> &sc, T stim, T dt,
                                          const double (&g)[TT_NEQ], double (&res)[ADJ_IN]) {
    using D = Dual<K, T>;
    D yd[TT_NEQ];
#pragma unroll
    for (int s = 0; s < TT_NEQ; ++s) {
        yd[s] = D(y[s]);
#pragma unroll
        for (int k = 0; k < K; ++k) yd[s].d[k] = (s == j0 + k) ? 1.0 : 0.0;
    }
    TTScale<D> sd;
    sd.gNa = D(sc.gNa);
    sd.gKr = D(sc.gKr);
    sd.gKs = D(sc.gKs);
    sd.gCaL = D(sc.gCaL);
    sd.gK1 = D(sc.gK1);
#pragma unroll
    for (int k = 0; k < K; ++k) sd.gKr.d[k] = (TT_NEQ == j0 + k) ? 1.0 : 0.0;
    const D dtd(dt);
    TTUpdate<D> u;
    tt2006_rhs<D>(yd, D(stim), dtd, sd, u);
    // the outputs of the sub-step, in the forms of k_tt2006_fp64
    D out[TT_NEQ];
    out[TT_V] = dtd * u.dV + yd[TT_V];
#pragma unroll
    for (int q = 0; q < 12; ++q) out[1 + q] = u.gate[q];
    out[TT_CAI] = dtd * u.dCai + yd[TT_CAI];
    out[TT_CASR] = dtd * u.dCaSR + yd[TT_CASR];
    out[TT_CASS] = dtd * u.dCaSS + yd[TT_CASS];
    out[TT_RPRIME] = dtd * u.dRprime + yd[TT_RPRIME];
    out[TT_NAI] = dtd * u.dNai + yd[TT_NAI];
    out[TT_KI] = dtd * u.dKi + yd[TT_KI];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (j0 + k >= ADJ_IN) break;
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < TT_NEQ; ++i) acc += g[i] * (double)out[i].d[k];
        res[j0 + k] = acc;
    }
}

// Per compact cell t: y = (v_n, s_n) from a snapshot, g = (alpha w, mu_in);
// writes lambda_n (grid), mu_out (state rows 1..18) and adds dL/dgKr.
template <int K>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_tt2006(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl_n,
                                                            const double *__restrict__ v_n,
                                                            const double *__restrict__ sv_n,
                                                            const double *__restrict__ w, double alpha,
                                                            const double *__restrict__ mu_in, double *mu_out,
                                                            double *lam_out, double *gth) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const size_t ld = o.ld;
    double y[TT_NEQ], gi[TT_NEQ];
    y[0] = v_n[g];
    gi[0] = alpha * w[g];
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) {
        y[s] = sv_n[s * ld + t];
        gi[s] = mu_in[s * ld + t];
    }
    const double stim = cell_stim(o, ctrl_n, t);
    const TTScale<double> sc = load_tt_scale<double>(o, t);
    double res[ADJ_IN];
    for (int j0 = 0; j0 < ADJ_IN; j0 += K) adj_block<K>(j0, y, sc, stim, o.dt, gi, res);
    lam_out[g] = res[0];
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) mu_out[s * ld + t] = res[s];
    gth[t] += res[TT_NEQ];
}

// The same for the mixed forward (k_tt2006_mixed): the state from the mixed
// rows of the snapshot (FP64 rows 1..5 = Ca_i, Ca_SR, Ca_ss, Na_i, K_i; FP32
// rows 0..11 = the gates, row 12 = R'), the Jacobian in FP32 dual numbers
// through the same model code, contracted and accumulated in FP64.
template <int K>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_tt2006_mixed(mb_ode_dev o, const mb_ctrl *__restrict__ ctrl_n,
                                                                  const double *__restrict__ v_n,
                                                                  const double *__restrict__ sv64_n,
                                                                  const float *__restrict__ sv32_n,
                                                                  const double *__restrict__ w, double alpha,
                                                                  const double *__restrict__ mu_in, double *mu_out,
                                                                  double *lam_out, double *gth) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= o.n) return;
    const uint32_t g = o.cell ? o.cell[t] : t;
    const size_t ld = o.ld;
    float y[TT_NEQ];
    double gi[TT_NEQ];
    y[TT_V] = (float)v_n[g];
#pragma unroll
    for (int k = 0; k < 12; ++k) y[1 + k] = sv32_n[k * ld + t];
    y[TT_CAI] = (float)sv64_n[1 * ld + t];
    y[TT_CASR] = (float)sv64_n[2 * ld + t];
    y[TT_CASS] = (float)sv64_n[3 * ld + t];
    y[TT_NAI] = (float)sv64_n[4 * ld + t];
    y[TT_KI] = (float)sv64_n[5 * ld + t];
    y[TT_RPRIME] = sv32_n[12 * ld + t];
    gi[0] = alpha * w[g];
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) gi[s] = mu_in[s * ld + t];
    const float stim = (float)cell_stim(o, ctrl_n, t);
    const TTScale<float> sc = load_tt_scale<float>(o, t);
    double res[ADJ_IN];
    for (int j0 = 0; j0 < ADJ_IN; j0 += K) adj_block<K, float>(j0, y, sc, stim, (float)o.dt, gi, res);
    lam_out[g] = res[0];
#pragma unroll
    for (int s = 1; s < TT_NEQ; ++s) mu_out[s * ld + t] = res[s];
    gth[t] += res[TT_NEQ];
}

// ---- conductivity gradient ---------------------------------------------------

// dL/dsigma_c += sum over the coupled faces of c of -(w_c - w_n)(v_c - v_n)
// m dH/dsigma_c, with H = 2 s_c s_n / (s_c + s_n) the face conductivity
// (fill_discretization_matrix_elements, assembly_common.c:969-991) and m the
// face's area / distance.
__global__ void k_adj_face_grad(mb_stencil_dev st, const double *__restrict__ sigma, const double *__restrict__ w,
                                const double *__restrict__ v, double mx, double my, double mz, double *gsig) {
    const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const unsigned m = st.code[g];
        if (!(m & 64u)) continue;
        const double sa = sigma[g], wa = w[g], va = v[g];
        const uint32_t nb[6] = {g - 1, g + 1, g - sy, g + sy, g - sz, g + sz};
        const double mult[6] = {mx, mx, my, my, mz, mz};
        double acc = 0.0;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            if (!((m >> q) & 1u)) continue;
            const double sb = sigma[nb[q]];
            if (sa == 0.0 || sb == 0.0) continue;
            const double s = sa + sb;
            const double dh = 2.0 * sb * sb / (s * s);
            acc += -(wa - w[nb[q]]) * (va - v[nb[q]]) * mult[q] * dh;
        }
        gsig[g] += acc;
    }
}

// ---- sensors, tolerance ----------------------------------------------------------

__global__ void k_adj_gather(const double *v, const int64_t *cells, int ns, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ns) out[i] = v[cells[i]];
}

__global__ void k_adj_scatter(double *lam, const int64_t *cells, int ns, const double *gsrc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ns) atomicAdd(&lam[cells[i]], gsrc[i]);
}

// tol of the transposed solve: rel^2 x (lambda . lambda) (one block, fixed
// summation order), floored so that an all-zero right-hand side stops at once.
__global__ void k_adj_tol(const double *lam, int64_t n, double rel2, mb_ctrl *c) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int64_t g = threadIdx.x; g < n; g += blockDim.x) s += lam[g] * lam[g];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) c->tol = c->refine_floor = fmax(rel2 * s, 1e-300);
    }
}

MB_NS_END

using namespace mb;

extern "C" int mbk_adj_tt2006(const mb_ode_dev *o, const mb_ctrl *ctrl_n, const double *v_n, const double *sv_n,
                              const double *w, double alpha, const double *mu_in, double *mu_out, double *lam_out,
                              double *gth, cudaStream_t s) {
    const unsigned blocks = (o->n + ADJ_THREADS - 1) / ADJ_THREADS;
    k_adj_tt2006<2><<<blocks, ADJ_THREADS, 0, s>>>(*o, ctrl_n, v_n, sv_n, w, alpha, mu_in, mu_out, lam_out, gth);
    return (int)cudaGetLastError();
}

extern "C" int mbk_adj_tt2006_mixed(const mb_ode_dev *o, const mb_ctrl *ctrl_n, const double *v_n,
                                    const double *sv64_n, const float *sv32_n, const double *w, double alpha,
                                    const double *mu_in, double *mu_out, double *lam_out, double *gth, cudaStream_t s) {
    const unsigned blocks = (o->n + ADJ_THREADS - 1) / ADJ_THREADS;
    k_adj_tt2006_mixed<2><<<blocks, ADJ_THREADS, 0, s>>>(*o, ctrl_n, v_n, sv64_n, sv32_n, w, alpha, mu_in, mu_out,
                                                        lam_out, gth);
    return (int)cudaGetLastError();
}

extern "C" int mbk_adj_face_grad(const mb_stencil_dev *st, const double *sigma, const double *w, const double *v,
                                 double mx, double my, double mz, double *gsig, cudaStream_t s) {
    k_adj_face_grad<<<592, 256, 0, s>>>(*st, sigma, w, v, mx, my, mz, gsig);
    return (int)cudaGetLastError();
}

extern "C" int mbk_adj_gather(const double *v, const int64_t *cells, int ns, double *out, cudaStream_t s) {
    k_adj_gather<<<(ns + 255) / 256, 256, 0, s>>>(v, cells, ns, out);
    return (int)cudaGetLastError();
}

extern "C" int mbk_adj_scatter(double *lam, const int64_t *cells, int ns, const double *gsrc, cudaStream_t s) {
    k_adj_scatter<<<(ns + 255) / 256, 256, 0, s>>>(lam, cells, ns, gsrc);
    return (int)cudaGetLastError();
}

extern "C" int mbk_adj_tol(const double *lam, int64_t n, double rel2, mb_ctrl *c, cudaStream_t s) {
    k_adj_tol<<<1, 1024, 0, s>>>(lam, n, rel2, c);
    return (int)cudaGetLastError();
}

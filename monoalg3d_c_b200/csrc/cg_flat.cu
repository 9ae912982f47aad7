// Persistent, cooperatively launched Jacobi-PCG: the whole CG solve of one
// time step is a single kernel.  Same recurrences and stopping rule as
// cpu_conjugate_gradient (src/linear_system_solver_library/linear_system_solver.c:47-183):
//   r = b - A x,  z = (1/diag) r,  p = z,  its = 1, error = r.r
//   while error >= tol and its < max_its:
//       alpha = r.z / p.Ap;  x += alpha p;  r -= alpha Ap
//       beta = r'.z' / r.z;  error = r'.r';  its += 1;  stop if error <= tol
//       p = z' + beta p
// with the right-hand side b = alpha_i V*_i formed in the first pass
// (update_monodomain.c:41-52).
//
// Per iteration the grid makes two passes over the cells, separated by grid
// reductions:
//   Q: p_new = z + beta p_old (evaluated for the cell and, on the fly, for its
//      stencil neighbours, so the direction update needs no pass of its own),
//      A p_new and the partial sums of p.Ap;
//   U: x += alpha p, r -= alpha A p (A p recomputed from p), z = r / diag and
//      the partial sums of r.z and r.r.
// p is double-buffered so Q reads p_old of neighbours while writing p_new.
// Every block adds the per-block partials in the same fixed order, so the
// scalars (alpha, beta, the stopping test) are bit-identical in every block.
//
// Mixed precision: p, r, z and A p in FP32, the solution x and every dot
// product in FP64; when the FP32 recurrence residual has dropped by
// refine_ratio (or below tol) the FP64 true residual b - A x replaces r and the
// iteration restarts from it; the stopping test uses that FP64 residual.
//
// Launch shapes are template parameters (threads per block, cells gathered
// per thread before use, per-cell or per-warp-row gathering); the host times
// the variants on the tissue's first solve and keeps the fastest.
#include <cstdint>
#include <type_traits>
#include <cuda/atomic>
#include <cuda_runtime.h>
#include "mb_internal.h"

namespace mb {
namespace fcg {

constexpr long long SPIN_LIMIT = 1LL << 24;   // bounded waits (about a second)

struct Args {
    mb_stencil_dev st;
    double *x;
    const double *vstar;
    const double *b;
    double *r64, *pa64, *pb64, *z64;
    float *r32, *pa32, *pb32, *z32;
    const double *inv_diag64;  // Jacobi 1/diag per cell (FP64 form)
    const float *inv_diag32;   // Jacobi 1/diag per cell (mixed form)
    double *partials;          // 2 x 4 x gridDim.x partials, then 2 x 4 totals
    mb_ctrl *ctrl;
    unsigned *bar;             // [0] arrivals, [1] generation
    int *status;
};

// Grid-wide sum of NV per-thread values.  Every block reduces its threads
// (warp shuffles, then one warp over the per-warp sums) and stores one
// partial per value; the block whose arrival completes the count (release
// atomic) adds the partials in block order -- a fixed order, so the totals are
// the same whichever block finishes last -- stores them and publishes a new
// generation (release store) that the other blocks wait for with acquire
// loads.  Partials and totals alternate between two buffers so a fast block
// never overwrites values a slow block has still to read.  Waits are bounded:
// after SPIN_LIMIT polls the block records MB_ERR_CUDA in the status word and
// returns false, and so does every block that later times out on it.
template <int NV, int NT>
__device__ __forceinline__ bool grid_reduce(const Args &a, double (&v)[NV], double (&out)[NV], int &red) {
    __shared__ double sm[NV][NT / 32];
    __shared__ double tot[NV];
    __shared__ int flag;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *part = a.partials + (size_t)(red & 1) * 4 * gridDim.x;
    double *total = a.partials + (size_t)8 * gridDim.x + (size_t)(red & 1) * 4;
    red++;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0) sm[q][warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> arrive(a.bar[0]);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(a.bar[1]);
        unsigned g0 = 0;
        int last = 0;
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = lane < NT / 32 ? sm[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) part[(size_t)q * gridDim.x + blockIdx.x] = s;
        }
        if (lane == 0) {
            g0 = gen.load(cuda::memory_order_relaxed);
            last = arrive.fetch_add(1u, cuda::memory_order_acq_rel) == gridDim.x - 1;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) {
            cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
#pragma unroll
            for (int q = 0; q < NV; ++q) {
                double s = 0.0;
                for (unsigned bk = lane; bk < gridDim.x; bk += 32) s += __ldcg(&part[(size_t)q * gridDim.x + bk]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                if (lane == 0) {
                    total[q] = s;
                    tot[q] = s;
                }
            }
            if (lane == 0) {
                arrive.store(0u, cuda::memory_order_relaxed);
                gen.store(g0 + 1u, cuda::memory_order_release);
                flag = 1;
            }
        } else if (lane == 0) {
            long long spins = 0;
            int ok = 1;
            while (gen.load(cuda::memory_order_acquire) == g0) {
                if (++spins > SPIN_LIMIT) {
                    atomicExch(a.status, MB_ERR_CUDA);
                    ok = 0;
                    break;
                }
                if (spins > 64) __nanosleep(20);
            }
            if (ok) {
#pragma unroll
                for (int q = 0; q < NV; ++q) tot[q] = __ldcg(&total[q]);
            }
            flag = ok ? 0 : 2;
        }
    }
    __syncthreads();
    if (flag == 2) return false;
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = tot[q];
    __syncthreads();
    return true;
}

// ---- operator rows ------------------------------------------------------------

__device__ __forceinline__ void cell_ijk(uint32_t g, uint32_t nx, uint32_t ny, int &i, int &j, int &k) {
    const uint32_t t = g / nx;
    i = (int)(g - t * nx);
    k = (int)(t / ny);
    j = (int)(t - (uint32_t)k * ny);
}

__device__ __forceinline__ bool active_at(const mb_stencil_dev &st, uint32_t g) {
    return st.mask == nullptr || st.mask[g] != 0;
}

// Diagonal of row (i,j,k): alpha plus every face coefficient, in the order
// -x, +x, -y, +y, -z, +z.
template <typename T>
__device__ __forceinline__ T diag_at(const mb_stencil_dev &st, int i, int j, int k, uint32_t g) {
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    if (st.kind == 0) {
        const uint8_t *m = st.mask;
        T dg = T(st.alpha);
        if (i > 0 && (!m || m[g - 1])) dg += T(st.cx);
        if (i < st.nx - 1 && (!m || m[g + 1])) dg += T(st.cx);
        if (j > 0 && (!m || m[g - sy])) dg += T(st.cy);
        if (j < st.ny - 1 && (!m || m[g + sy])) dg += T(st.cy);
        if (k > 0 && (!m || m[g - sz])) dg += T(st.cz);
        if (k < st.nz - 1 && (!m || m[g + sz])) dg += T(st.cz);
        return dg;
    } else if (st.kind == 1) {
        T dg = T(st.alpha);
        if (i > 0) dg += T(st.fx[g - 1]);
        if (i < st.nx - 1) dg += T(st.fx[g]);
        if (j > 0) dg += T(st.fy[g - sy]);
        if (j < st.ny - 1) dg += T(st.fy[g]);
        if (k > 0) dg += T(st.fz[g - sz]);
        if (k < st.nz - 1) dg += T(st.fz[g]);
        return dg;
    } else {
        const int cxk = (i == 0) ? 0 : (i == st.nx - 1 ? 2 : 1);
        const int cyk = (j == 0) ? 0 : (j == st.ny - 1 ? 2 : 1);
        const size_t row = ((size_t)k * 9 + cyk * 3 + cxk) * 27;
        return sizeof(T) == 8 ? T(st.table[row + 13]) : T(st.table32[row + 13]);
    }
}

// A 7-point row gathered for one cell: the field at the cell and its six
// neighbours (-x, +x, -y, +y, -z, +z; clamped to the cell outside the domain,
// where the coupling is zero) and which faces couple (bit q of m); kind 1
// also carries the six face coefficients.  Removed cells hold zeros in every
// vector, so every load of a row can be issued before the mask is known.
template <typename T, int KIND>
struct Row7 {
    T pc, p[6];
    T c[KIND == 1 ? 6 : 1];
    unsigned m;
    bool on;
};

template <typename T, int KIND, typename PF>
__device__ __forceinline__ Row7<T, KIND> gather_cell(const mb_stencil_dev &st, uint32_t g, PF pf) {
    Row7<T, KIND> R;
    int i, j, k;
    cell_ijk(g, st.nx, st.ny, i, j, k);
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    const bool v0 = i > 0, v1 = i < st.nx - 1, v2 = j > 0, v3 = j < st.ny - 1, v4 = k > 0, v5 = k < st.nz - 1;
    const uint32_t n0 = v0 ? g - 1 : g, n1 = v1 ? g + 1 : g, n2 = v2 ? g - sy : g, n3 = v3 ? g + sy : g;
    const uint32_t n4 = v4 ? g - sz : g, n5 = v5 ? g + sz : g;
    R.pc = pf(g);
    R.p[0] = pf(n0); R.p[1] = pf(n1); R.p[2] = pf(n2); R.p[3] = pf(n3); R.p[4] = pf(n4); R.p[5] = pf(n5);
    R.on = active_at(st, g);
    if constexpr (KIND == 0) {
        const uint8_t *mk = st.mask;
        unsigned m = (unsigned)v0 | ((unsigned)v1 << 1) | ((unsigned)v2 << 2) | ((unsigned)v3 << 3) |
                     ((unsigned)v4 << 4) | ((unsigned)v5 << 5);
        if (mk) {
            m &= (unsigned)(mk[n0] != 0) | ((unsigned)(mk[n1] != 0) << 1) | ((unsigned)(mk[n2] != 0) << 2) |
                 ((unsigned)(mk[n3] != 0) << 3) | ((unsigned)(mk[n4] != 0) << 4) | ((unsigned)(mk[n5] != 0) << 5);
        }
        R.m = m;
    } else {
        R.c[0] = v0 ? T(st.fx[n0]) : T(0); R.c[1] = T(st.fx[g]);
        R.c[2] = v2 ? T(st.fy[n2]) : T(0); R.c[3] = T(st.fy[g]);
        R.c[4] = v4 ? T(st.fz[n4]) : T(0); R.c[5] = T(st.fz[g]);
        R.m = 0x3f;
    }
    return R;
}

// The same row for lane l of a warp segment (32 consecutive cells of an
// x-row): the +-x neighbours come from the adjacent lanes by shuffles (only
// lanes 0 and 31 read memory for them).  Lanes past the end of the row work on
// a clamped copy and are marked inactive.
template <typename T, int KIND, typename PF>
__device__ __forceinline__ Row7<T, KIND> gather_seg(const mb_stencil_dev &st, uint32_t unit, uint32_t nseg, PF pf,
                                                    uint32_t &gout) {
    const int lane = threadIdx.x & 31;
    const uint32_t row = unit / nseg, seg = unit - row * nseg;
    const int k = (int)(row / (uint32_t)st.ny), j = (int)(row - (uint32_t)k * st.ny);
    const int i = (int)seg * 32 + lane;
    const bool valid = i < st.nx;
    const int ic = valid ? i : st.nx - 1;
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    const uint32_t g = row * (uint32_t)st.nx + (uint32_t)ic;
    gout = g;
    const bool v0 = ic > 0, v1 = ic < st.nx - 1, v2 = j > 0, v3 = j < st.ny - 1, v4 = k > 0, v5 = k < st.nz - 1;
    const uint32_t n2 = v2 ? g - sy : g, n3 = v3 ? g + sy : g, n4 = v4 ? g - sz : g, n5 = v5 ? g + sz : g;
    Row7<T, KIND> R;
    R.pc = pf(g);
    R.p[2] = pf(n2);
    R.p[3] = pf(n3);
    R.p[4] = pf(n4);
    R.p[5] = pf(n5);
    T left = __shfl_up_sync(0xffffffffu, R.pc, 1);
    T right = __shfl_down_sync(0xffffffffu, R.pc, 1);
    if (lane == 0) left = pf(v0 ? g - 1 : g);
    if (lane == 31) right = pf(v1 ? g + 1 : g);
    R.p[0] = left;
    R.p[1] = right;
    const uint8_t *mk = st.mask;
    const unsigned self_on = mk ? (mk[g] != 0) : 1u;
    R.on = valid && self_on;
    if constexpr (KIND == 0) {
        unsigned m = (unsigned)v0 | ((unsigned)v1 << 1) | ((unsigned)v2 << 2) | ((unsigned)v3 << 3) |
                     ((unsigned)v4 << 4) | ((unsigned)v5 << 5);
        if (mk) {
            unsigned ml = __shfl_up_sync(0xffffffffu, self_on, 1);
            unsigned mr = __shfl_down_sync(0xffffffffu, self_on, 1);
            if (lane == 0) ml = v0 ? (mk[g - 1] != 0) : 0u;
            if (lane == 31) mr = v1 ? (mk[g + 1] != 0) : 0u;
            m &= ml | (mr << 1) | ((unsigned)(mk[n2] != 0) << 2) | ((unsigned)(mk[n3] != 0) << 3) |
                 ((unsigned)(mk[n4] != 0) << 4) | ((unsigned)(mk[n5] != 0) << 5);
        }
        R.m = m;
    } else {
        const T fxg = T(st.fx[g]);
        T fxl = __shfl_up_sync(0xffffffffu, fxg, 1);
        if (lane == 0) fxl = v0 ? T(st.fx[g - 1]) : T(0);
        R.c[0] = v0 ? fxl : T(0);
        R.c[1] = fxg;
        R.c[2] = v2 ? T(st.fy[n2]) : T(0);
        R.c[3] = T(st.fy[g]);
        R.c[4] = v4 ? T(st.fz[n4]) : T(0);
        R.c[5] = T(st.fz[g]);
        R.m = 0x3f;
    }
    return R;
}

// (A p)_c from a gathered 7-point row: alpha p_c + sum c (p_c - p_n), in the
// reference's row order.
template <typename T, int KIND>
__device__ __forceinline__ T row_apply(const mb_stencil_dev &st, const Row7<T, KIND> &R) {
    T acc = T(st.alpha) * R.pc;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        T c;
        if constexpr (KIND == 0) c = (R.m >> q) & 1u ? T(q < 2 ? st.cx : (q < 4 ? st.cy : st.cz)) : T(0);
        else c = R.c[q];
        acc += c * (R.pc - R.p[q]);
    }
    return R.on ? acc : T(0);
}

// 27-point rows (kind 2) from the per-plane class table; the product is
// formed while gathering.  Coefficients of missing neighbours are zero and
// their loads are clamped to the cell.
template <typename T>
struct Row27 {
    T pc, ap;
    bool on;
};

template <typename T, typename PF>
__device__ __forceinline__ Row27<T> gather27(const mb_stencil_dev &st, uint32_t g, PF pf) {
    Row27<T> R;
    int i, j, k;
    cell_ijk(g, st.nx, st.ny, i, j, k);
    R.on = active_at(st, g);
    R.pc = pf(g);
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    const int cxk = (i == 0) ? 0 : (i == st.nx - 1 ? 2 : 1);
    const int cyk = (j == 0) ? 0 : (j == st.ny - 1 ? 2 : 1);
    const size_t row = ((size_t)k * 9 + cyk * 3 + cxk) * 27;
    T acc = T(0);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const int q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                const T c = sizeof(T) == 8 ? T(st.table[row + q]) : T(st.table32[row + q]);
                if (q == 13) {
                    acc += c * R.pc;
                } else {
                    const uint32_t gn = c != T(0) ? g + dx + (int)sy * dy + (int)sz * dz : g;
                    acc += c * pf(gn);
                }
            }
    R.ap = R.on ? acc : T(0);
    return R;
}

// ---- sweeps ------------------------------------------------------------------

// Contiguous, warp-aligned range of cells owned by this block.
__device__ __forceinline__ void block_chunk(uint32_t n, uint32_t &c0, uint32_t &c1) {
    const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 31u) & ~31u;
    c0 = min(n, blockIdx.x * chunk);
    c1 = min(n, c0 + chunk);
}

// Cell sweep: each thread takes U cells of the block's range at a time and
// gathers all U rows (their loads in flight together) before using them.
template <int NT, int U, typename G, typename C>
__device__ __forceinline__ void cell_sweep(uint32_t c0, uint32_t c1, G gather, C compute) {
    for (uint32_t base = c0 + threadIdx.x; base < c1; base += U * NT) {
        decltype(gather(0u)) rows[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t g = base + u * NT;
            rows[u] = gather(g < c1 ? g : base);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t g = base + u * NT;
            if (g < c1 && rows[u].on) compute(g, rows[u]);
        }
    }
}

// Segment sweep: each warp takes U 32-cell row segments of the block's range
// at a time.
template <typename T, int KIND, int NT, int U, typename PF, typename ACT>
__device__ __forceinline__ void seg_sweep(const mb_stencil_dev &st, PF pf, ACT act) {
    constexpr int WARPS = NT / 32;
    const uint32_t nseg = (uint32_t)(st.nx + 31) / 32;
    const uint32_t units = nseg * (uint32_t)st.ny * (uint32_t)st.nz;
    const uint32_t per = (units + gridDim.x - 1) / gridDim.x;
    const uint32_t u0 = min(units, blockIdx.x * per), u1 = min(units, u0 + per);
    const int warp = threadIdx.x >> 5;
    for (uint32_t base = u0 + warp; base < u1; base += U * WARPS) {
        Row7<T, KIND> rows[U];
        uint32_t gs[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t unit = base + u * WARPS;
            rows[u] = gather_seg<T, KIND>(st, unit < u1 ? unit : base, nseg, pf, gs[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t unit = base + u * WARPS;
            if (unit < u1 && rows[u].on) act(gs[u], rows[u]);
        }
    }
}

// A pass over all active cells for any operator kind and launch shape.
template <typename T, int KIND, int NT, int U, bool SEG, typename PF, typename ACT>
__device__ __forceinline__ void pass(const mb_stencil_dev &st, PF pf, ACT act) {
    if constexpr (KIND != 2 && SEG) {
        seg_sweep<T, KIND, NT, U>(st, pf, act);
    } else {
        const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
        uint32_t c0, c1;
        block_chunk(n, c0, c1);
        if constexpr (KIND == 2)
            cell_sweep<NT, U>(c0, c1, [&](uint32_t g) { return gather27<T>(st, g, pf); }, act);
        else
            cell_sweep<NT, U>(c0, c1, [&](uint32_t g) { return gather_cell<T, KIND>(st, g, pf); }, act);
    }
}

template <typename T, int KIND, typename R>
__device__ __forceinline__ T product(const mb_stencil_dev &st, const R &row) {
    if constexpr (KIND == 2) return row.ap;
    else return row_apply<T, KIND>(st, row);
}

// ---- the solve ----------------------------------------------------------------

template <bool MIXED>
struct Prec { using T = double; };
template <>
struct Prec<true> { using T = float; };

template <bool MIXED>
__device__ __forceinline__ typename Prec<MIXED>::T inv_d(const Args &a, uint32_t g) {
    if constexpr (MIXED) return a.inv_diag32[g];
    else return a.inv_diag64[g];
}

// FP64 true residual r = b - A x; stores r (in T), z and p = z; accumulates
// r.z (T products, FP64 sums), r.r of the stored r, and the FP64 r.r.
template <bool MIXED, int KIND, int NT, int U, bool SEG>
__device__ __forceinline__ void residual_pass(const Args &a, typename Prec<MIXED>::T *r,
                                              typename Prec<MIXED>::T *p, bool pre, double (&acc)[3]) {
    using T = typename Prec<MIXED>::T;
    const mb_stencil_dev &st = a.st;
    const double *__restrict__ x = a.x;
    pass<double, KIND, NT, U, SEG>(st, [&](uint32_t q) { return x[q]; },
                                  [&](uint32_t g, const auto &row) {
                                      const double ax = product<double, KIND>(st, row);
                                      const double bb = a.b ? a.b[g] : st.alpha * a.vstar[g];
                                      const double r64 = bb - ax;
                                      const T rt = (T)r64;
                                      const T z = pre ? inv_d<MIXED>(a, g) * rt : rt;
                                      r[g] = rt;
                                      p[g] = z;
                                      acc[0] += (double)rt * (double)z;
                                      acc[1] += (double)rt * (double)rt;
                                      acc[2] += r64 * r64;
                                  });
}

template <bool MIXED, int KIND, int NT, int U, bool SEG>
__global__ void __launch_bounds__(NT, 1) k_fcg(Args a) {
    using T = typename Prec<MIXED>::T;
    const mb_stencil_dev &st = a.st;
    mb_ctrl *c = a.ctrl;
    const bool pre = c->use_precond != 0;
    const double tol = c->tol;
    const int max_its = c->max_its;
    const double ratio = c->refine_ratio;
    T *__restrict__ r = MIXED ? (T *)a.r32 : (T *)a.r64;
    T *__restrict__ zb = MIXED ? (T *)a.z32 : (T *)a.z64;
    T *bufa = MIXED ? (T *)a.pa32 : (T *)a.pa64;
    T *bufb = MIXED ? (T *)a.pb32 : (T *)a.pb64;
    int red = 0;

    double acc[3] = {0.0, 0.0, 0.0}, s3[3];
    residual_pass<MIXED, KIND, NT, U, SEG>(a, r, bufa, pre, acc);
    if (!grid_reduce<3, NT>(a, acc, s3, red)) return;
    double rz = s3[0], rr = s3[1];
    double error = s3[2], rr_ref = s3[2];
    int its = 1, refinements = MIXED ? 1 : 0;
    bool done = !(s3[2] >= tol) || !(1 < max_its);
    bool first = true;
    double beta = 0.0;
    T *pold = bufa, *pnew = bufb;

    while (!done) {
        // Q: direction p_new = z + beta p_old fused with A p_new and p.Ap
        T *pcur = first ? pold : pnew;
        const T *__restrict__ po = pold;
        T *__restrict__ pw = pnew;
        const T bt = (T)beta;
        double q1[1] = {0.0}, s1[1];
        if (first) {
            pass<T, KIND, NT, U, SEG>(st, [&](uint32_t q) { return po[q]; },
                                      [&](uint32_t g, const auto &row) {
                                          q1[0] += (double)row.pc * (double)product<T, KIND>(st, row);
                                      });
        } else {
            pass<T, KIND, NT, U, SEG>(st, [&](uint32_t q) { return zb[q] + bt * po[q]; },
                                      [&](uint32_t g, const auto &row) {
                                          pw[g] = row.pc;
                                          q1[0] += (double)row.pc * (double)product<T, KIND>(st, row);
                                      });
        }
        if (!grid_reduce<1, NT>(a, q1, s1, red)) return;
        const double alpha = (pre ? rz : rr) / s1[0];
        const T al = (T)alpha;

        // U: x += alpha p, r -= alpha A p, z = r / diag
        double u2[2] = {0.0, 0.0}, s2[2];
        const T *__restrict__ pc_ = pcur;
        double *__restrict__ x = a.x;
        pass<T, KIND, NT, U, SEG>(st, [&](uint32_t q) { return pc_[q]; },
                                  [&](uint32_t g, const auto &row) {
                                      const T ap = product<T, KIND>(st, row);
                                      x[g] += alpha * (double)row.pc;
                                      const T rn = r[g] - al * ap;
                                      r[g] = rn;
                                      const T z = pre ? inv_d<MIXED>(a, g) * rn : rn;
                                      zb[g] = z;
                                      u2[0] += (double)z * (double)rn;
                                      u2[1] += (double)rn * (double)rn;
                                  });
        if (!grid_reduce<2, NT>(a, u2, s2, red)) return;
        its += 1;
        pold = pcur;
        pnew = (pcur == bufa) ? bufb : bufa;
        if (!MIXED) {
            const double b_next = pre ? s2[0] / rz : s2[1] / rr;
            error = s2[1];
            if (s2[1] <= tol || its >= max_its) {
                done = true;
            } else {
                beta = b_next;
                rz = s2[0];
                rr = s2[1];
                first = false;
            }
        } else {
            if (s2[1] <= fmax(tol, ratio * rr_ref) || its >= max_its) {
                // FP64 true residual replaces the FP32 recurrence; restart from it
                double t3[3] = {0.0, 0.0, 0.0};
                residual_pass<MIXED, KIND, NT, U, SEG>(a, r, pold, pre, t3);
                if (!grid_reduce<3, NT>(a, t3, s3, red)) return;
                refinements += 1;
                error = s3[2];
                rr_ref = s3[2];
                rz = s3[0];
                rr = s3[1];
                first = true;
                if (s3[2] <= tol || its >= max_its) done = true;
            } else {
                beta = pre ? s2[0] / rz : s2[1] / rr;
                rz = s2[0];
                rr = s2[1];
                error = s2[1];
                first = false;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->its = its;
        c->error = error;
        c->refinements = refinements;
        c->rz = rz;
        c->rr = rr;
        c->done = 1;
    }
}

// Jacobi inverse diagonal 1/diag per active cell, computed once per operator
// (the reference forms (1.0 / elements[0].value) at each use; the value is the same).
__global__ void k_inv_diag(mb_stencil_dev st, double *d64, float *d32) {
    const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        if (!active_at(st, g)) continue;
        int i, j, k;
        cell_ijk(g, st.nx, st.ny, i, j, k);
        if (d64) d64[g] = 1.0 / diag_at<double>(st, i, j, k, g);
        if (d32) d32[g] = 1.0f / diag_at<float>(st, i, j, k, g);
    }
}

// ---- variants -------------------------------------------------------------------

struct Variant {
    const void *fn;
    int threads;
};

template <bool MIXED, int KIND>
struct Table;

#define MB_V(NT, U, SEG) {(const void *)k_fcg<MIXED, KIND, NT, U, SEG>, NT}
template <bool MIXED>
struct Table<MIXED, 0> {
    static constexpr int KIND = 0;
    static constexpr int N = 5;
    static Variant get(int v) {
        const Variant t[N] = {MB_V(1024, 1, false), MB_V(1024, 1, true), MB_V(512, 2, false), MB_V(512, 2, true),
                              MB_V(512, 4, false)};
        return t[v];
    }
};
template <bool MIXED>
struct Table<MIXED, 1> {
    static constexpr int KIND = 1;
    static constexpr int N = 3;
    static Variant get(int v) {
        const Variant t[N] = {MB_V(1024, 1, false), MB_V(1024, 1, true), MB_V(512, 2, false)};
        return t[v];
    }
};
template <bool MIXED>
struct Table<MIXED, 2> {
    static constexpr int KIND = 2;
    static constexpr int N = 2;
    static Variant get(int v) {
        const Variant t[N] = {MB_V(1024, 1, false), MB_V(512, 1, false)};
        return t[v];
    }
};
#undef MB_V

static Variant variant(int mixed, int kind, int v) {
    if (mixed) {
        if (kind == 0) return Table<true, 0>::get(v);
        if (kind == 1) return Table<true, 1>::get(v);
        return Table<true, 2>::get(v);
    }
    if (kind == 0) return Table<false, 0>::get(v);
    if (kind == 1) return Table<false, 1>::get(v);
    return Table<false, 2>::get(v);
}

}  // namespace fcg
}  // namespace mb

using namespace mb::fcg;

extern "C" int mbk_fcg_variants(int kind) {
    return kind == 0 ? Table<false, 0>::N : (kind == 1 ? Table<false, 1>::N : Table<false, 2>::N);
}

// Co-resident blocks of a variant (the grid size of its cooperative launch).
extern "C" int mbk_fcg_max_blocks(int mixed, int kind, int v) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    const Variant var = variant(mixed, kind, v);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, var.fn, var.threads, 0) != cudaSuccess) return -1;
    return sms * per;
}

extern "C" int mbk_inv_diag(const mb_stencil_dev *st, double *d64, float *d32, cudaStream_t s) {
    k_inv_diag<<<592, 256, 0, s>>>(*st, d64, d32);
    return (int)cudaGetLastError();
}

extern "C" int mbk_fcg_launch(const mb_pcg_dev *p, cudaStream_t s) {
    Args a;
    a.st = p->st;
    a.x = p->x; a.vstar = p->vstar; a.b = p->b;
    a.r64 = p->r64; a.pa64 = p->pa64; a.pb64 = p->pb64; a.z64 = p->z64;
    a.r32 = p->r32; a.pa32 = p->pa32; a.pb32 = p->pb32; a.z32 = p->z32;
    a.inv_diag64 = p->inv_diag64; a.inv_diag32 = p->inv_diag32;
    a.partials = p->partials; a.ctrl = p->ctrl; a.bar = p->bar; a.status = p->status;
    const Variant var = variant(p->mixed, p->st.kind, p->variant);
    void *args[] = {&a};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p->blocks);
    cfg.blockDim = dim3(var.threads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelExC(&cfg, var.fn, args);
}

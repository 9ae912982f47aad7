// Jacobi-preconditioned conjugate gradient on the structured monodomain
// operator (alpha I + K), matrix-free.
//
// Recurrences and stopping rule follow cpu_conjugate_gradient
// (src/linear_system_solver_library/linear_system_solver.c:47-183):
//   r = b - A x,  z = (1/diag) r,  p = z,  its = 1, error = r.r
//   while error >= tol and its < max_its:
//       alpha = r.z / p.Ap;  x += alpha p;  r -= alpha Ap
//       beta = r'.z' / r.z;  error = r'.r';  its += 1;  stop if error <= tol
//       p = z' + beta p
// with b = alpha_i V*_i formed inside the first kernel (update_monodomain.c:41-52).
//
// Layout: every vector is indexed by the grid index g = i + nx (j + ny k).
// Each iteration is three grid-stride kernels (p.Ap; x/r update; new
// direction); A p is recomputed from p where it is needed instead of being
// stored.  Dot products are reduced per block with warp shuffles and shared
// memory, then summed in a fixed order by the last block to finish, which also
// evaluates the scalar recurrences and the stopping rule on the device and
// sets the condition of the CUDA-graph WHILE node that repeats the iteration.
//
// Mixed precision: p, r and A p in FP32, the solution x and every dot product
// in FP64; when the FP32 recurrence residual has dropped by refine_ratio (or
// below tol) the FP64 true residual b - A x is evaluated, replaces r, and the
// iteration restarts from it; the stopping rule is applied to that FP64
// residual only.
#include <cstdint>
#include <cuda_runtime.h>
#include "mb_internal.h"

namespace mb {

constexpr int CG_THREADS = 256;

struct CgArgs {
    mb_stencil_dev st;
    mb_cg_dev cg;
    mb_ctrl *ctrl;
    unsigned long long cond;
    int use_cond;
};

__device__ __forceinline__ void decompose(int64_t g, int nx, int ny, int &i, int &j, int &k) {
    const int64_t t = g / nx;
    i = (int)(g - t * nx);
    k = (int)(t / ny);
    j = (int)(t - (int64_t)k * ny);
}

__device__ __forceinline__ bool is_active(const mb_stencil_dev &st, int64_t g) {
    return st.mask == nullptr || st.mask[g] != 0;
}

// (A p)_g and the diagonal of row g, with A = alpha I + K; K is assembled
// with no flux across the domain boundary or into removed cells
// (assembly_common.c:911-1048).  Written as alpha p_g + sum c (p_g - p_n).
template <typename T>
__device__ __forceinline__ T apply_row(const mb_stencil_dev &st, const T *__restrict__ p, int i, int j, int k,
                                       int64_t g, T &diag) {
    const T pc = p[g];
    const int64_t sx = 1, sy = st.nx, sz = (int64_t)st.nx * st.ny;
    if (st.kind == 0) {
        T acc = T(st.alpha) * pc;
        T dg = T(st.alpha);
        const T cx = T(st.cx), cy = T(st.cy), cz = T(st.cz);
        const uint8_t *m = st.mask;
#define MB_NB(cond, off, c)                                        \
        if ((cond) && (m == nullptr || m[g + (off)])) {            \
            dg += (c);                                             \
            acc += (c) * (pc - p[g + (off)]);                      \
        }
        MB_NB(i > 0, -sx, cx)
        MB_NB(i < st.nx - 1, sx, cx)
        MB_NB(j > 0, -sy, cy)
        MB_NB(j < st.ny - 1, sy, cy)
        MB_NB(k > 0, -sz, cz)
        MB_NB(k < st.nz - 1, sz, cz)
#undef MB_NB
        diag = dg;
        return acc;
    } else if (st.kind == 1) {
        T acc = T(st.alpha) * pc;
        T dg = T(st.alpha);
#define MB_FC(cond, off, c)                                        \
        if (cond) {                                                \
            const T cc = T(c);                                     \
            dg += cc;                                              \
            acc += cc * (pc - p[g + (off)]);                       \
        }
        MB_FC(i > 0, -sx, st.fx[g - sx])
        MB_FC(i < st.nx - 1, sx, st.fx[g])
        MB_FC(j > 0, -sy, st.fy[g - sy])
        MB_FC(j < st.ny - 1, sy, st.fy[g])
        MB_FC(k > 0, -sz, st.fz[g - sz])
        MB_FC(k < st.nz - 1, sz, st.fz[g])
#undef MB_FC
        diag = dg;
        return acc;
    } else {
        // 27-point rows from the class table: class = (k, x boundary, y boundary)
        const int cxk = (i == 0) ? 0 : (i == st.nx - 1 ? 2 : 1);
        const int cyk = (j == 0) ? 0 : (j == st.ny - 1 ? 2 : 1);
        const size_t row = ((size_t)k * 9 + cyk * 3 + cxk) * 27;
        T acc = T(0);
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    const int n = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                    T c;
                    if (sizeof(T) == 8) c = T(st.table[row + n]);
                    else c = T(st.table32[row + n]);
                    if (c != T(0)) acc += c * p[g + dx * sx + dy * sy + dz * sz];
                }
            }
        }
        if (sizeof(T) == 8) diag = T(st.table[row + 13]);
        else diag = T(st.table32[row + 13]);
        return acc;
    }
}

// Diagonal only (used by the direction update).
template <typename T>
__device__ __forceinline__ T row_diag(const mb_stencil_dev &st, int i, int j, int k, int64_t g) {
    const int64_t sx = 1, sy = st.nx, sz = (int64_t)st.nx * st.ny;
    if (st.kind == 0) {
        T dg = T(st.alpha);
        const uint8_t *m = st.mask;
        if (i > 0 && (!m || m[g - sx])) dg += T(st.cx);
        if (i < st.nx - 1 && (!m || m[g + sx])) dg += T(st.cx);
        if (j > 0 && (!m || m[g - sy])) dg += T(st.cy);
        if (j < st.ny - 1 && (!m || m[g + sy])) dg += T(st.cy);
        if (k > 0 && (!m || m[g - sz])) dg += T(st.cz);
        if (k < st.nz - 1 && (!m || m[g + sz])) dg += T(st.cz);
        return dg;
    } else if (st.kind == 1) {
        T dg = T(st.alpha);
        if (i > 0) dg += T(st.fx[g - sx]);
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

// ---- reductions -----------------------------------------------------------

// Block-reduce NV doubles and store them as this block's partials.
template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double *partials) {
    __shared__ double sm[NV][CG_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if (lane == 0) sm[q][warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = lane < CG_THREADS / 32 ? sm[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) partials[q * gridDim.x + blockIdx.x] = s;
        }
    }
}

// True in every thread of the block that finished last.  Resets the ticket.
__device__ __forceinline__ bool finish_last(mb_ctrl *c) {
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(&c->ticket, 1u);
        last = (t == gridDim.x - 1);
        if (last) c->ticket = 0;
    }
    __syncthreads();
    if (last) __threadfence();
    return last != 0;
}

// Fixed-order sum of the NV partial arrays, valid in thread 0 of the last block.
template <int NV>
__device__ __forceinline__ void sum_partials(const double *partials, double (&out)[NV]) {
    __shared__ double sm[NV][CG_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
        for (unsigned b = threadIdx.x; b < gridDim.x; b += CG_THREADS) s += __ldcg(&partials[q * gridDim.x + b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) sm[q][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (int w = 0; w < CG_THREADS / 32; ++w) s += sm[q][w];
            out[q] = s;
        }
    }
}

__device__ __forceinline__ void set_cond(const CgArgs &a, bool cont) {
    if (a.use_cond) cudaGraphSetConditional(a.cond, cont ? 1u : 0u);
}

// ---- FP64 -------------------------------------------------------------------

__global__ void __launch_bounds__(CG_THREADS) k_cg64_init(CgArgs a) {
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const bool pre = a.ctrl->use_precond != 0;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    double acc[2] = {0.0, 0.0};
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        int i, j, k;
        decompose(g, st.nx, st.ny, i, j, k);
        double dg;
        const double ax = apply_row<double>(st, cg.x, i, j, k, g, dg);
        const double b = cg.b ? cg.b[g] : st.alpha * cg.vstar[g];
        const double r = b - ax;
        const double z = pre ? (1.0 / dg) * r : r;
        cg.r[g] = r;
        cg.p[g] = z;
        acc[0] += r * z;
        acc[1] += r * r;
    }
    block_partials<2>(acc, cg.partials);
    if (finish_last(a.ctrl)) {
        double s[2];
        sum_partials<2>(cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->rz = s[0];
            c->rr = s[1];
            c->error = s[1];
            c->its = 1;
            c->refinements = 0;
            c->phase = 0;
            c->done = !(s[1] >= c->tol) || !(1 < c->max_its);
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cg64_pq(CgArgs a) {
    if (a.ctrl->done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(a, false);
        return;
    }
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    double acc[1] = {0.0};
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        int i, j, k;
        decompose(g, st.nx, st.ny, i, j, k);
        double dg;
        const double ap = apply_row<double>(st, cg.p, i, j, k, g, dg);
        acc[0] += cg.p[g] * ap;
    }
    block_partials<1>(acc, cg.partials);
    if (finish_last(a.ctrl)) {
        double s[1];
        sum_partials<1>(cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->pq = s[0];
            c->alpha = (c->use_precond ? c->rz : c->rr) / s[0];
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cg64_update(CgArgs a) {
    if (a.ctrl->done) return;
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const bool pre = a.ctrl->use_precond != 0;
    const double alpha = a.ctrl->alpha;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    double acc[2] = {0.0, 0.0};
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        int i, j, k;
        decompose(g, st.nx, st.ny, i, j, k);
        double dg;
        const double ap = apply_row<double>(st, cg.p, i, j, k, g, dg);
        cg.x[g] += alpha * cg.p[g];
        const double r = cg.r[g] - alpha * ap;
        cg.r[g] = r;
        const double z = pre ? (1.0 / dg) * r : r;
        acc[0] += z * r;
        acc[1] += r * r;
    }
    block_partials<2>(acc, cg.partials);
    if (finish_last(a.ctrl)) {
        double s[2];
        sum_partials<2>(cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            const double beta = c->use_precond ? s[0] / c->rz : s[1] / c->rr;
            c->error = s[1];
            c->its += 1;
            if (s[1] <= c->tol || c->its >= c->max_its) {
                c->done = 1;
            } else {
                c->beta = beta;
                c->rz = s[0];
                c->rr = s[1];
            }
            set_cond(a, !c->done);
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cg64_dir(CgArgs a) {
    if (a.ctrl->done) return;
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const bool pre = a.ctrl->use_precond != 0;
    const double beta = a.ctrl->beta;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        const double r = cg.r[g];
        double z = r;
        if (pre) {
            int i, j, k;
            decompose(g, st.nx, st.ny, i, j, k);
            z = (1.0 / row_diag<double>(st, i, j, k, g)) * r;
        }
        cg.p[g] = z + beta * cg.p[g];
    }
}

// ---- mixed precision ------------------------------------------------------

// FP64 true residual r = b - A x into r32; p32 = z; accumulates r.r (FP64),
// and r32.z (FP64 accumulation of FP32 products).
__device__ __forceinline__ void mixed_residual_pass(const CgArgs &a, double (&acc)[3]) {
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const bool pre = a.ctrl->use_precond != 0;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        int i, j, k;
        decompose(g, st.nx, st.ny, i, j, k);
        double dg;
        const double ax = apply_row<double>(st, cg.x, i, j, k, g, dg);
        const double b = cg.b ? cg.b[g] : st.alpha * cg.vstar[g];
        const double r = b - ax;
        const float r32 = (float)r;
        const float z = pre ? (1.0f / (float)dg) * r32 : r32;
        cg.r32[g] = r32;
        cg.p32[g] = z;
        acc[0] += (double)r32 * (double)z;
        acc[1] += r * r;
        acc[2] += (double)r32 * (double)r32;
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cgm_init(CgArgs a) {
    double acc[3] = {0.0, 0.0, 0.0};
    mixed_residual_pass(a, acc);
    block_partials<3>(acc, a.cg.partials);
    if (finish_last(a.ctrl)) {
        double s[3];
        sum_partials<3>(a.cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->rz = s[0];
            c->rr = s[2];
            c->rr_ref = s[1];
            c->error = s[1];
            c->its = 1;
            c->refinements = 1;
            c->phase = 0;
            c->done = !(s[1] >= c->tol) || !(1 < c->max_its);
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cgm_pq(CgArgs a) {
    if (a.ctrl->done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(a, false);
        return;
    }
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    double acc[1] = {0.0};
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        int i, j, k;
        decompose(g, st.nx, st.ny, i, j, k);
        float dg;
        const float ap = apply_row<float>(st, cg.p32, i, j, k, g, dg);
        acc[0] += (double)cg.p32[g] * (double)ap;
    }
    block_partials<1>(acc, cg.partials);
    if (finish_last(a.ctrl)) {
        double s[1];
        sum_partials<1>(cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->pq = s[0];
            c->alpha = (c->use_precond ? c->rz : c->rr) / s[0];
            if (c->phase == 2) c->phase = 0;
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cgm_update(CgArgs a) {
    if (a.ctrl->done) return;
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const bool pre = a.ctrl->use_precond != 0;
    const double alpha = a.ctrl->alpha;
    const float alphaf = (float)alpha;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    double acc[2] = {0.0, 0.0};
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        int i, j, k;
        decompose(g, st.nx, st.ny, i, j, k);
        float dg;
        const float ap = apply_row<float>(st, cg.p32, i, j, k, g, dg);
        const float p = cg.p32[g];
        cg.x[g] += alpha * (double)p;
        const float r = cg.r32[g] - alphaf * ap;
        cg.r32[g] = r;
        const float z = pre ? (1.0f / dg) * r : r;
        acc[0] += (double)z * (double)r;
        acc[1] += (double)r * (double)r;
    }
    block_partials<2>(acc, cg.partials);
    if (finish_last(a.ctrl)) {
        double s[2];
        sum_partials<2>(cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->its += 1;
            const double lim = fmax(c->refine_floor, c->refine_ratio * c->rr_ref);
            if (s[1] <= lim) {
                c->phase = 1;                 // evaluate the FP64 residual next
            } else if (c->its >= c->max_its) {
                c->phase = 1;                 // final FP64 residual for the error
            } else {
                c->beta = c->use_precond ? s[0] / c->rz : s[1] / c->rr;
                c->rz = s[0];
                c->rr = s[1];
                c->error = s[1];
            }
            set_cond(a, true);
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cgm_refine(CgArgs a) {
    if (a.ctrl->done || a.ctrl->phase != 1) return;
    double acc[3] = {0.0, 0.0, 0.0};
    mixed_residual_pass(a, acc);
    block_partials<3>(acc, a.cg.partials);
    if (finish_last(a.ctrl)) {
        double s[3];
        sum_partials<3>(a.cg.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->refinements += 1;
            c->error = s[1];
            c->rr_ref = s[1];
            c->rz = s[0];
            c->rr = s[2];
            c->phase = 2;                     // restart: keep p = z this iteration
            if (s[1] <= c->tol || c->its >= c->max_its) c->done = 1;
            set_cond(a, !c->done);
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_cgm_dir(CgArgs a) {
    if (a.ctrl->done || a.ctrl->phase != 0) return;
    const mb_stencil_dev &st = a.st;
    const mb_cg_dev &cg = a.cg;
    const bool pre = a.ctrl->use_precond != 0;
    const float beta = (float)a.ctrl->beta;
    const int64_t n = (int64_t)st.nx * st.ny * st.nz;
    for (int64_t g = (int64_t)blockIdx.x * CG_THREADS + threadIdx.x; g < n; g += (int64_t)gridDim.x * CG_THREADS) {
        if (!is_active(st, g)) continue;
        const float r = cg.r32[g];
        float z = r;
        if (pre) {
            int i, j, k;
            decompose(g, st.nx, st.ny, i, j, k);
            z = (1.0f / row_diag<float>(st, i, j, k, g)) * r;
        }
        cg.p32[g] = z + beta * cg.p32[g];
    }
}

// ---- end of a loop step -------------------------------------------------

// Records the CG result, flags NaN, shifts periodic stimuli
// (ode_solver.c:225-233) and advances the loop clock
// (monodomain_solver.c:907-908).
__global__ void k_step_end(mb_ctrl *c, double dt_pde, double dt_ode, int num_steps, mb_step_stats *log,
                           int64_t log_len) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (log && c->count >= 0 && c->count < log_len) {
        mb_step_stats s;
        s.cg_iterations = c->its;
        s.refinements = c->refinements;
        s.cg_error = c->error;
        log[c->count] = s;
    }
    if (isnan(c->error)) c->nan_flag = 1;
    double time = c->cur_time;
    for (int j = 0; j < num_steps; ++j) time += dt_ode;
    for (int k = 0; k < c->num_stims; ++k) {
        if (c->stim_period[k] > 0.0 && time >= c->stim_start[k] + c->stim_period[k])
            c->stim_start[k] = c->stim_start[k] + c->stim_period[k];
    }
    c->count += 1;
    c->cur_time += dt_pde;
}

__global__ void k_set_nan(double *v, const uint8_t *mask, int64_t n) {
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x)
        if (mask && !mask[g]) v[g] = __longlong_as_double(0x7ff8000000000000LL);
}

// ---- general CSR CG (matrices read from file) ----------------------------

struct CsrArgs {
    mb_csr_dev m;
    mb_ctrl *ctrl;
};

__global__ void __launch_bounds__(CG_THREADS) k_csr_init(CsrArgs a) {
    const mb_csr_dev &m = a.m;
    const bool pre = a.ctrl->use_precond != 0;
    double acc[2] = {0.0, 0.0};
    for (int row = blockIdx.x * CG_THREADS + threadIdx.x; row < m.n; row += gridDim.x * CG_THREADS) {
        double ax = 0.0, dg = 0.0;
        for (int e = m.row_ptr[row]; e < m.row_ptr[row + 1]; ++e) {
            ax += m.val[e] * m.x[m.col[e]];
            if (m.col[e] == row) dg = m.val[e];
        }
        if (dg == 0.0) dg = 1.0;
        m.inv_diag[row] = 1.0 / dg;
        const double r = m.b[row] - ax;
        const double z = pre ? m.inv_diag[row] * r : r;
        m.r[row] = r;
        m.p[row] = z;
        acc[0] += r * z;
        acc[1] += r * r;
    }
    block_partials<2>(acc, m.partials);
    if (finish_last(a.ctrl)) {
        double s[2];
        sum_partials<2>(m.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->rz = s[0];
            c->rr = s[1];
            c->error = s[1];
            c->its = 1;
            c->done = !(s[1] >= c->tol) || !(1 < c->max_its);
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_csr_pq(CsrArgs a) {
    if (a.ctrl->done) return;
    const mb_csr_dev &m = a.m;
    double acc[1] = {0.0};
    for (int row = blockIdx.x * CG_THREADS + threadIdx.x; row < m.n; row += gridDim.x * CG_THREADS) {
        double q = 0.0;
        for (int e = m.row_ptr[row]; e < m.row_ptr[row + 1]; ++e) q += m.val[e] * m.p[m.col[e]];
        m.q[row] = q;
        acc[0] += m.p[row] * q;
    }
    block_partials<1>(acc, m.partials);
    if (finish_last(a.ctrl)) {
        double s[1];
        sum_partials<1>(m.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            c->alpha = (c->use_precond ? c->rz : c->rr) / s[0];
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_csr_update(CsrArgs a) {
    if (a.ctrl->done) return;
    const mb_csr_dev &m = a.m;
    const bool pre = a.ctrl->use_precond != 0;
    const double alpha = a.ctrl->alpha;
    double acc[2] = {0.0, 0.0};
    for (int row = blockIdx.x * CG_THREADS + threadIdx.x; row < m.n; row += gridDim.x * CG_THREADS) {
        m.x[row] += alpha * m.p[row];
        const double r = m.r[row] - alpha * m.q[row];
        m.r[row] = r;
        const double z = pre ? m.inv_diag[row] * r : r;
        acc[0] += z * r;
        acc[1] += r * r;
    }
    block_partials<2>(acc, m.partials);
    if (finish_last(a.ctrl)) {
        double s[2];
        sum_partials<2>(m.partials, s);
        if (threadIdx.x == 0) {
            mb_ctrl *c = a.ctrl;
            const double beta = c->use_precond ? s[0] / c->rz : s[1] / c->rr;
            c->error = s[1];
            c->its += 1;
            if (s[1] <= c->tol || c->its >= c->max_its) {
                c->done = 1;
            } else {
                c->beta = beta;
                c->rz = s[0];
                c->rr = s[1];
            }
        }
    }
}

__global__ void __launch_bounds__(CG_THREADS) k_csr_dir(CsrArgs a) {
    if (a.ctrl->done) return;
    const mb_csr_dev &m = a.m;
    const bool pre = a.ctrl->use_precond != 0;
    const double beta = a.ctrl->beta;
    for (int row = blockIdx.x * CG_THREADS + threadIdx.x; row < m.n; row += gridDim.x * CG_THREADS) {
        const double r = m.r[row];
        const double z = pre ? m.inv_diag[row] * r : r;
        m.p[row] = z + beta * m.p[row];
    }
}

}  // namespace mb

using namespace mb;

// Blocks of the graph-form CG kernels and the CSR kernels' partial-sum
// arrays: 8 per SM of the current device (looked up once per device).
extern "C" int mbk_max_grid_blocks(void) {
    static int per_device[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148 * 8;
    }
    if (!per_device[dev]) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            sms = 148;
        }
        per_device[dev] = sms * 8;
    }
    return per_device[dev];
}

extern "C" int mbk_cg_init(const mb_stencil_dev *st, const mb_cg_dev *cg, mb_ctrl *ctrl, unsigned long long cond,
                           int use_cond, cudaStream_t s) {
    CgArgs a{*st, *cg, ctrl, cond, use_cond};
    if (cg->precision == MB_PREC_FP64) k_cg64_init<<<cg->grid_blocks, CG_THREADS, 0, s>>>(a);
    else k_cgm_init<<<cg->grid_blocks, CG_THREADS, 0, s>>>(a);
    return (int)cudaGetLastError();
}

extern "C" int mbk_cg_body(const mb_stencil_dev *st, const mb_cg_dev *cg, mb_ctrl *ctrl, unsigned long long cond,
                           int use_cond, cudaStream_t s) {
    CgArgs a{*st, *cg, ctrl, cond, use_cond};
    const int gb = cg->grid_blocks;
    if (cg->precision == MB_PREC_FP64) {
        k_cg64_pq<<<gb, CG_THREADS, 0, s>>>(a);
        k_cg64_update<<<gb, CG_THREADS, 0, s>>>(a);
        k_cg64_dir<<<gb, CG_THREADS, 0, s>>>(a);
    } else {
        k_cgm_pq<<<gb, CG_THREADS, 0, s>>>(a);
        k_cgm_update<<<gb, CG_THREADS, 0, s>>>(a);
        k_cgm_refine<<<gb, CG_THREADS, 0, s>>>(a);
        k_cgm_dir<<<gb, CG_THREADS, 0, s>>>(a);
    }
    return (int)cudaGetLastError();
}

extern "C" int mbk_step_end(mb_ctrl *ctrl, double dt_pde, double dt_ode, int num_steps, mb_step_stats *log,
                            int64_t log_len, cudaStream_t s) {
    k_step_end<<<1, 32, 0, s>>>(ctrl, dt_pde, dt_ode, num_steps, log, log_len);
    return (int)cudaGetLastError();
}

extern "C" int mbk_set_nan(double *v, const uint8_t *mask, int64_t n, cudaStream_t s) {
    if (!mask || n == 0) return 0;
    k_set_nan<<<296, 256, 0, s>>>(v, mask, n);
    return (int)cudaGetLastError();
}

extern "C" int mbk_csr_cg_init(const mb_csr_dev *m, mb_ctrl *ctrl, cudaStream_t s) {
    CsrArgs a{*m, ctrl};
    k_csr_init<<<m->grid_blocks, CG_THREADS, 0, s>>>(a);
    return (int)cudaGetLastError();
}

extern "C" int mbk_csr_cg_iter(const mb_csr_dev *m, mb_ctrl *ctrl, cudaStream_t s) {
    CsrArgs a{*m, ctrl};
    k_csr_pq<<<m->grid_blocks, CG_THREADS, 0, s>>>(a);
    k_csr_update<<<m->grid_blocks, CG_THREADS, 0, s>>>(a);
    k_csr_dir<<<m->grid_blocks, CG_THREADS, 0, s>>>(a);
    return (int)cudaGetLastError();
}

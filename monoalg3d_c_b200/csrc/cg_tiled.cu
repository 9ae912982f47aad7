// Persistent Jacobi-PCG with 2.5D tiling: the same solve as cg_flat.cu
// (recurrences and stopping rule of cpu_conjugate_gradient,
// linear_system_solver.c:47-183; b = alpha V* fused, update_monodomain.c:41-52)
// but every pass streams the grid as tiles of 30 x 14 cells marching in z.
//
// A block is 32 x 16 threads; thread (tx, ty) owns column (i0 - 1 + tx,
// j0 - 1 + ty), so the outer ring of threads covers the one-cell halo.  For
// each plane the block computes the pass's input field once per cell (for the
// direction pass p_new = z + beta p_old from r, 1/diag and p_old) into one of
// three shared-memory planes, then the interior threads apply the 7-point or
// 27-point row from the planes k-1, k, k+1.  Each field value is loaded from
// global memory once per tile (plus the halo), instead of once per neighbour
// use.  Work items are (tile, z-chunk) pairs handed to the persistent blocks in
// a fixed order; the grid reductions use a bounded barrier (the last block
// to arrive adds the partials and publishes a new generation).
#include <cstdint>
#include <type_traits>
#include <cuda/atomic>
#include <cuda_runtime.h>
#include "mb_internal.h"

namespace mb {
namespace tcg {

constexpr int BX = 32, BY = 16;            // block = tile + halo
constexpr int TX = BX - 2, TY = BY - 2;    // interior cells per plane
constexpr int THREADS = BX * BY;
constexpr long long SPIN_LIMIT = 1LL << 24;

struct Args {
    mb_stencil_dev st;
    double *x;
    const double *vstar;
    const double *b;
    double *r64, *pa64, *pb64;
    float *r32, *pa32, *pb32;
    const double *inv_diag64;
    const float *inv_diag32;
    double *partials;       // 2 x 4 x gridDim.x partials, then 2 x 4 totals
    mb_ctrl *ctrl;
    unsigned *bar;          // [0] arrivals, [1] generation
    int *status;
    int tiles_x, tiles_y, zchunk, nchunks;
};

// Grid-wide sum: fixed-order sum of block partials by the last block to
// arrive, release/acquire generation word, bounded wait.
template <int NV>
__device__ __forceinline__ bool grid_reduce(const Args &a, double (&v)[NV], double (&out)[NV], int &red) {
    __shared__ double sm[NV][THREADS / 32];
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
            double s = lane < THREADS / 32 ? sm[q][lane] : 0.0;
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

template <bool MIXED>
struct Prec { using T = double; };
template <>
struct Prec<true> { using T = float; };

template <bool MIXED>
__device__ __forceinline__ typename Prec<MIXED>::T inv_d(const Args &a, uint32_t g) {
    if constexpr (MIXED) return a.inv_diag32[g];
    else return a.inv_diag64[g];
}

// Shared planes: 3 planes of field values (as F) and of cell activity.
template <typename F>
struct Planes {
    F v[3][BY][BX];
    uint8_t on[3][BY][BX];
};

// Geometry of the thread's column within the current work item.
struct Col {
    int i, j;          // grid coordinates of the column
    bool inside;       // column inside the grid
    bool interior;     // thread applies the row (not a halo thread)
    uint32_t g0;       // grid index at k = 0
};

__device__ __forceinline__ Col column(const Args &a, int item, int &z0, int &z1) {
    const int tiles = a.tiles_x * a.tiles_y;
    const int tile = item % tiles, zc = item / tiles;
    const int txi = tile % a.tiles_x, tyi = tile / a.tiles_x;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    Col c;
    c.i = txi * TX - 1 + tx;
    c.j = tyi * TY - 1 + ty;
    c.inside = c.i >= 0 && c.i < a.st.nx && c.j >= 0 && c.j < a.st.ny;
    c.interior = c.inside && tx >= 1 && tx <= TX && ty >= 1 && ty <= TY;
    c.g0 = c.inside ? (uint32_t)c.i + (uint32_t)a.st.nx * (uint32_t)c.j : 0u;
    z0 = zc * a.zchunk;
    z1 = min(a.st.nz, z0 + a.zchunk);
    return c;
}

// (A P)_c at interior thread (tx, ty), plane slots km, kc, kp.
template <typename T, typename F>
__device__ __forceinline__ T stencil(const Args &a, const Planes<F> &P, int km, int kc, int kp, const Col &c, int k,
                                     uint32_t g) {
    const mb_stencil_dev &st = a.st;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const T pc = (T)P.v[kc][ty][tx];
    if (st.kind == 0) {
        const T cx = T(st.cx), cy = T(st.cy), cz = T(st.cz), zero = T(0);
        const T c0 = P.on[kc][ty][tx - 1] ? cx : zero, c1 = P.on[kc][ty][tx + 1] ? cx : zero;
        const T c2 = P.on[kc][ty - 1][tx] ? cy : zero, c3 = P.on[kc][ty + 1][tx] ? cy : zero;
        const T c4 = P.on[km][ty][tx] ? cz : zero, c5 = P.on[kp][ty][tx] ? cz : zero;
        T acc = T(st.alpha) * pc;
        acc += c0 * (pc - (T)P.v[kc][ty][tx - 1]);
        acc += c1 * (pc - (T)P.v[kc][ty][tx + 1]);
        acc += c2 * (pc - (T)P.v[kc][ty - 1][tx]);
        acc += c3 * (pc - (T)P.v[kc][ty + 1][tx]);
        acc += c4 * (pc - (T)P.v[km][ty][tx]);
        acc += c5 * (pc - (T)P.v[kp][ty][tx]);
        return acc;
    } else if (st.kind == 1) {
        const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
        const T c0 = c.i > 0 ? T(st.fx[g - 1]) : T(0), c1 = T(st.fx[g]);
        const T c2 = c.j > 0 ? T(st.fy[g - sy]) : T(0), c3 = T(st.fy[g]);
        const T c4 = k > 0 ? T(st.fz[g - sz]) : T(0), c5 = T(st.fz[g]);
        T acc = T(st.alpha) * pc;
        acc += c0 * (pc - (T)P.v[kc][ty][tx - 1]);
        acc += c1 * (pc - (T)P.v[kc][ty][tx + 1]);
        acc += c2 * (pc - (T)P.v[kc][ty - 1][tx]);
        acc += c3 * (pc - (T)P.v[kc][ty + 1][tx]);
        acc += c4 * (pc - (T)P.v[km][ty][tx]);
        acc += c5 * (pc - (T)P.v[kp][ty][tx]);
        return acc;
    } else {
        const int cxk = (c.i == 0) ? 0 : (c.i == st.nx - 1 ? 2 : 1);
        const int cyk = (c.j == 0) ? 0 : (c.j == st.ny - 1 ? 2 : 1);
        const size_t row = ((size_t)k * 9 + cyk * 3 + cxk) * 27;
        const int slot[3] = {km, kc, kp};
        T acc = T(0);
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    const int q = dz * 9 + dy * 3 + dx;
                    const T cf = sizeof(T) == 8 ? T(st.table[row + q]) : T(st.table32[row + q]);
                    acc += cf * (T)P.v[slot[dz]][ty - 1 + dy][tx - 1 + dx];
                }
        return acc;
    }
}

// One pass over every work item.  load(g) gives the pass's input field at an
// active cell; act(...) runs at every active interior cell once planes k-1,
// k, k+1 are in shared memory.
template <typename F, typename LOAD, typename ACT>
__device__ __forceinline__ void sweep(const Args &a, Planes<F> &P, LOAD load, ACT act) {
    const mb_stencil_dev &st = a.st;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int nitems = a.tiles_x * a.tiles_y * a.nchunks;
    const uint32_t nxy = (uint32_t)st.nx * st.ny;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        int z0, z1;
        const Col c = column(a, item, z0, z1);
        auto fill = [&](int k, int slot) {
            F val = F(0);
            uint8_t on = 0;
            if (c.inside && k >= 0 && k < st.nz) {
                const uint32_t g = c.g0 + (uint32_t)k * nxy;
                on = st.mask ? st.mask[g] : (uint8_t)1;
                if (on) val = load(g);
            }
            P.v[slot][ty][tx] = val;
            P.on[slot][ty][tx] = on;
        };
        fill(z0 - 1, (z0 + 2) % 3);
        fill(z0, z0 % 3);
        for (int k = z0; k < z1; ++k) {
            fill(k + 1, (k + 1) % 3);
            __syncthreads();
            const int kc = k % 3;
            if (c.interior && P.on[kc][ty][tx]) act(c, k, c.g0 + (uint32_t)k * nxy, (k + 2) % 3, kc, (k + 1) % 3);
            __syncthreads();
        }
    }
}

// FP64 true residual r = b - A x, p = z; sums r.z, r.r (stored r), r.r (FP64).
template <bool MIXED>
__device__ __forceinline__ void residual_pass(const Args &a, unsigned char *smem, typename Prec<MIXED>::T *r,
                                              typename Prec<MIXED>::T *p, bool pre, double (&acc)[3]) {
    using T = typename Prec<MIXED>::T;
    Planes<double> &P = *reinterpret_cast<Planes<double> *>(smem);
    sweep<double>(a, P, [&](uint32_t g) { return a.x[g]; },
                  [&](const Col &c, int k, uint32_t g, int km, int kc, int kp) {
                      const double ax = stencil<double, double>(a, P, km, kc, kp, c, k, g);
                      const double bb = a.b ? a.b[g] : a.st.alpha * a.vstar[g];
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

template <bool MIXED>
__global__ void __launch_bounds__(THREADS, 2) k_tcg(Args a) {
    using T = typename Prec<MIXED>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    Planes<T> &P = *reinterpret_cast<Planes<T> *>(smem);
    mb_ctrl *c = a.ctrl;
    const bool pre = c->use_precond != 0;
    const double tol = c->tol;
    const int max_its = c->max_its;
    const double ratio = c->refine_ratio;
    T *r = MIXED ? (T *)a.r32 : (T *)a.r64;
    T *bufa = MIXED ? (T *)a.pa32 : (T *)a.pa64;
    T *bufb = MIXED ? (T *)a.pb32 : (T *)a.pb64;
    int red = 0;

    double acc[3] = {0.0, 0.0, 0.0}, s3[3];
    residual_pass<MIXED>(a, smem, r, bufa, pre, acc);
    if (!grid_reduce<3>(a, acc, s3, red)) return;
    double rz = s3[0], rr = s3[1];
    double error = s3[2], rr_ref = s3[2];
    int its = 1, refinements = MIXED ? 1 : 0;
    bool done = !(s3[2] >= tol) || !(1 < max_its);
    bool first = true;
    double beta = 0.0;
    T *pold = bufa, *pnew = bufb;

    while (!done) {
        // Q: p_new = z + beta p_old on the planes, A p_new, p.Ap
        T *pcur = first ? pold : pnew;
        const T bt = (T)beta;
        double q1[1] = {0.0}, s1[1];
        if (first) {
            sweep<T>(a, P, [&](uint32_t g) { return pold[g]; },
                     [&](const Col &cc, int k, uint32_t g, int km, int kc, int kp) {
                         const T pc = P.v[kc][threadIdx.x >> 5][threadIdx.x & 31];
                         const T ap = stencil<T, T>(a, P, km, kc, kp, cc, k, g);
                         q1[0] += (double)pc * (double)ap;
                     });
        } else {
            sweep<T>(a, P,
                     [&](uint32_t g) {
                         const T rq = r[g];
                         const T z = pre ? inv_d<MIXED>(a, g) * rq : rq;
                         return z + bt * pold[g];
                     },
                     [&](const Col &cc, int k, uint32_t g, int km, int kc, int kp) {
                         const T pc = P.v[kc][threadIdx.x >> 5][threadIdx.x & 31];
                         pnew[g] = pc;
                         const T ap = stencil<T, T>(a, P, km, kc, kp, cc, k, g);
                         q1[0] += (double)pc * (double)ap;
                     });
        }
        if (!grid_reduce<1>(a, q1, s1, red)) return;
        const double alpha = (pre ? rz : rr) / s1[0];
        const T al = (T)alpha;

        // U: x += alpha p, r -= alpha A p
        double u2[2] = {0.0, 0.0}, s2[2];
        sweep<T>(a, P, [&](uint32_t g) { return pcur[g]; },
                 [&](const Col &cc, int k, uint32_t g, int km, int kc, int kp) {
                     const T pc = P.v[kc][threadIdx.x >> 5][threadIdx.x & 31];
                     const T ap = stencil<T, T>(a, P, km, kc, kp, cc, k, g);
                     a.x[g] += alpha * (double)pc;
                     const T rn = r[g] - al * ap;
                     r[g] = rn;
                     const T z = pre ? inv_d<MIXED>(a, g) * rn : rn;
                     u2[0] += (double)z * (double)rn;
                     u2[1] += (double)rn * (double)rn;
                 });
        if (!grid_reduce<2>(a, u2, s2, red)) return;
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
            if (s2[1] <= fmax(c->refine_floor, ratio * rr_ref) || its >= max_its) {
                double t3[3] = {0.0, 0.0, 0.0};
                residual_pass<MIXED>(a, smem, r, pold, pre, t3);
                if (!grid_reduce<3>(a, t3, s3, red)) return;
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

}  // namespace tcg
}  // namespace mb

using namespace mb::tcg;

static size_t tcg_smem() { return sizeof(Planes<double>); }

extern "C" int mbk_tcg_max_blocks(int mixed) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    cudaError_t e = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tcg<true>, THREADS, tcg_smem())
                          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tcg<false>, THREADS, tcg_smem());
    if (e != cudaSuccess) return -1;
    return sms * per;
}

// Tiles of the grid and the z-chunk length that give at least `blocks` work
// items with the fewest extra halo planes.
extern "C" void mbk_tcg_layout(int nx, int ny, int nz, int blocks, int *tiles_x, int *tiles_y, int *zchunk,
                               int *nchunks) {
    const int tx = (nx + TX - 1) / TX, ty = (ny + TY - 1) / TY;
    const int tiles = tx * ty;
    int best_zc = nz;
    double best = 1e30;
    for (int zc = 1; zc <= nz; ++zc) {
        const int nc = (nz + zc - 1) / zc;
        const long items = (long)tiles * nc;
        const long waves = (items + blocks - 1) / blocks;
        // cost ~ per-block planes on the critical path: waves x (zc + 2 halo planes)
        const double cost = (double)waves * (zc + 2);
        if (cost < best) { best = cost; best_zc = zc; }
    }
    *tiles_x = tx;
    *tiles_y = ty;
    *zchunk = best_zc;
    *nchunks = (nz + best_zc - 1) / best_zc;
}

extern "C" int mbk_tcg_launch(const mb_pcg_dev *p, cudaStream_t s) {
    Args a;
    a.st = p->st;
    a.x = p->x; a.vstar = p->vstar; a.b = p->b;
    a.r64 = p->r64; a.pa64 = p->pa64; a.pb64 = p->pb64;
    a.r32 = p->r32; a.pa32 = p->pa32; a.pb32 = p->pb32;
    a.inv_diag64 = p->inv_diag64; a.inv_diag32 = p->inv_diag32;
    a.partials = p->partials; a.ctrl = p->ctrl; a.bar = p->bar; a.status = p->status;
    a.tiles_x = p->tiles_x; a.tiles_y = p->tiles_y; a.zchunk = p->zchunk; a.nchunks = p->nchunks;
    // the barrier words start from zero in every launch
    cudaError_t e = cudaMemsetAsync(p->bar, 0, 2 * sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    void *args[] = {&a};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p->blocks);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = tcg_smem();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const void *fn = p->mixed ? (const void *)k_tcg<true> : (const void *)k_tcg<false>;
    return (int)cudaLaunchKernelExC(&cfg, fn, args);
}

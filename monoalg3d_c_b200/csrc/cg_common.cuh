// Pieces shared by the persistent CG kernels (cg_flat.cu, cg_resident.cu):
// the launch arguments and the bounded grid-wide reduction.
#pragma once
#include <cstdint>
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
    double *ap64;              // A p of the current direction (stored by Q, read by U)
    float *ap32;
    float *ap32b;              // the z-march fused pass's second A p buffer
    double *w;                 // the z-march fused solve's stored A x (FP64), or NULL
    const double *inv_diag64;  // Jacobi 1/diag per cell (FP64 form)
    const float *inv_diag32;   // Jacobi 1/diag per cell (mixed form)
    double *partials;          // 2 x 8 x gridDim.x partials
    mb_ctrl *ctrl;
    unsigned *bar;             // [0] arrivals since launch (zeroed before each launch)
    int *status;
};

// Grid-wide sum of NV per-thread values.  Every block reduces its threads
// (warp shuffles, then one warp over the per-warp sums), stores its partials
// and counts its arrival (release).  The arrival counter only grows during a
// launch: the r-th reduction is complete when it reaches (r + 1) x blocks.
// Each block then adds all partials itself, in block order and with the same
// shuffle tree, so every block holds bit-identical totals without a second
// hand-off.  Partials alternate between two buffers, so a fast block never
// overwrites values a slow block has still to read.  Waits are bounded: after
// SPIN_LIMIT polls the block records MB_ERR_CUDA in the status word and
// returns false (the caller leaves the kernel).
template <int NV, int NT>
__device__ __forceinline__ bool grid_reduce(const Args &a, double (&v)[NV], double (&out)[NV], int &red) {
    static_assert(NV >= 1 && NV <= 8, "the partials hold up to 8 values per block");
    // partials loaded per lane before the adds (fewer for many values)
    constexpr int J = NV <= 4 ? 8 : 4;
    __shared__ double sm[NV][NT / 32];
    __shared__ double tot[NV];
    __shared__ int flag;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *part = a.partials + (size_t)(red & 1) * 8 * gridDim.x;
    const unsigned target = (unsigned)(red + 1) * gridDim.x;
    red++;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        if (lane == 0) sm[q][warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> arrive(a.bar[0]);
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = lane < (int)(blockDim.x >> 5) ? sm[q][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) part[(size_t)q * gridDim.x + blockIdx.x] = s;
        }
        int ok = 1;
        if (lane == 0) {
            arrive.fetch_add(1u, cuda::memory_order_release);
            long long spins = 0;
            while (arrive.load(cuda::memory_order_acquire) < target) {
                if (++spins > SPIN_LIMIT) {
                    atomicExch(a.status, MB_ERR_CUDA);
                    ok = 0;
                    break;
                }
                if (spins > 4096) __nanosleep(32);
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        // every lane that reads the partials orders its reads after the
        // arrivals lane 0 observed
        cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
        if (ok) {
            // every partial of a chunk of up to 32 J blocks is loaded before
            // any is added, so the reads cost one L2 round trip, not one per value
            double s[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) s[q] = 0.0;
            for (unsigned base = 0; base < gridDim.x; base += 32 * J) {
                double vals[NV][J];
#pragma unroll
                for (int q = 0; q < NV; ++q)
#pragma unroll
                    for (int j = 0; j < J; ++j) {
                        const unsigned bk = base + lane + 32 * j;
                        vals[q][j] = bk < gridDim.x ? __ldcg(&part[(size_t)q * gridDim.x + bk]) : 0.0;
                    }
#pragma unroll
                for (int q = 0; q < NV; ++q)
#pragma unroll
                    for (int j = 0; j < J; ++j) s[q] += vals[q][j];
            }
#pragma unroll
            for (int q = 0; q < NV; ++q) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
                if (lane == 0) tot[q] = s[q];
            }
        }
        if (lane == 0) flag = ok;
    }
    __syncthreads();
    if (!flag) return false;
    // tot, sm and flag are next written only after the next reduction's first
    // __syncthreads, which every thread reaches after reading them here
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = tot[q];
    return true;
}

// bit 6 of a cell's code byte: the cell is active
constexpr unsigned ACTIVE = 64u;

}  // namespace fcg
}  // namespace mb

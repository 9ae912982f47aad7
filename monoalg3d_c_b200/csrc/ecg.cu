// Pseudo-bidomain ECG on the device, the computation of the reference's
// pseudo_bidomain_cpu (ecg_library/ecg.c:204-307) with the divergence
// matrix of assembly_divergent / fill_element (ecg.c:36-43, 149-172):
//   per active cell, each face neighbour that is an active cell inside the
//   domain carries value_ecg = -m and the diagonal +m, m = dx dy / dz for
//   every face direction;
//   beta_im = sum(value_ecg v) / vol, cell after cell;
//   lead_l = -(1 / (4 pi sigma_b)) sum_cells beta_im / |x_cell - lead_l| vol.
// The distances are formed on the fly from the cell centres instead of being
// stored (n_leads x cells doubles in the reference).  Two launches: per-block
// partial sums of every lead, then one block that adds them in block order
// (so the result does not depend on scheduling) and appends the record.
// Both return at once on steps that take no record.
#include <cstdint>
#include <cuda_runtime.h>
#include "mb_internal.h"

namespace mb {
namespace ecg {

constexpr int NT = 256;
constexpr unsigned ACTIVE = 64u;   // bit 6 of a code byte: the cell is active

__device__ __forceinline__ bool record_step(const mb_ctrl *c, const mb_ecg_dev &e) {
    return e.rate > 0 && (c->count % e.rate) == 0 && c->ecg_count < e.capacity;
}

__global__ void __launch_bounds__(NT) k_ecg_partials(mb_stencil_dev st, const double *__restrict__ v, mb_ecg_dev e,
                                                     const mb_ctrl *__restrict__ c) {
    if (!record_step(c, e)) return;
    const int nl = e.n_leads;
    const uint32_t nx = st.nx, ny = st.ny, nz = st.nz;
    const uint32_t sy = nx, sz = nx * ny, n = sz * nz;
    const double m = (e.dx * e.dy) / e.dz, vol = e.dx * e.dy * e.dz;
    double acc[MB_ECG_MAX_LEADS];
#pragma unroll
    for (int l = 0; l < MB_ECG_MAX_LEADS; ++l) acc[l] = 0.0;
    for (uint32_t g = blockIdx.x * NT + threadIdx.x; g < n; g += gridDim.x * NT) {
        const uint32_t i = g % nx, t = g / nx, j = t % ny, k = t / ny;
        unsigned bits;
        if (st.code) {
            bits = st.code[g];
        } else {
            bits = ACTIVE | (i > 0 ? 1u : 0u) | (i + 1 < nx ? 2u : 0u) | (j > 0 ? 4u : 0u) | (j + 1 < ny ? 8u : 0u) |
                   (k > 0 ? 16u : 0u) | (k + 1 < nz ? 32u : 0u);
        }
        if (!(bits & ACTIVE)) continue;
        const double vc = v[g];
        double beta = (__popc(bits & 63u) * m) * vc / vol;
        if (bits & 1u) beta += -m * v[g - 1] / vol;
        if (bits & 2u) beta += -m * v[g + 1] / vol;
        if (bits & 4u) beta += -m * v[g - sy] / vol;
        if (bits & 8u) beta += -m * v[g + sy] / vol;
        if (bits & 16u) beta += -m * v[g - sz] / vol;
        if (bits & 32u) beta += -m * v[g + sz] / vol;
        const double cx = (i + 0.5) * e.dx, cy = (j + 0.5) * e.dy, cz = (k + 0.5) * e.dz;
#pragma unroll
        for (int l = 0; l < MB_ECG_MAX_LEADS; ++l) {
            if (l >= nl) break;
            const double ex = e.leads[3 * l] - cx, ey = e.leads[3 * l + 1] - cy, ez = e.leads[3 * l + 2] - cz;
            const double dist = sqrt(ex * ex + ey * ey + ez * ez);
            acc[l] += beta / dist * vol;
        }
    }
    __shared__ double sm[MB_ECG_MAX_LEADS][NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int l = 0; l < MB_ECG_MAX_LEADS; ++l) {
        if (l >= nl) break;
        double s = acc[l];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sm[l][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < (unsigned)nl) {
        double s = 0.0;
        for (int w = 0; w < NT / 32; ++w) s += sm[threadIdx.x][w];
        e.partials[(size_t)blockIdx.x * MB_ECG_MAX_LEADS + threadIdx.x] = s;
    }
}

__global__ void k_ecg_finish(mb_ecg_dev e, mb_ctrl *c, int nblocks) {
    if (!record_step(c, e)) return;
    const int nl = e.n_leads;
    const int64_t rec = c->ecg_count;
    double *row = e.log + (size_t)rec * (1 + nl);
    if (threadIdx.x < (unsigned)nl) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += e.partials[(size_t)b * MB_ECG_MAX_LEADS + threadIdx.x];
        row[1 + threadIdx.x] = -e.scale * s;
    }
    if (threadIdx.x == 0) row[0] = c->cur_time;
    __syncthreads();   // every thread has read ecg_count
    if (threadIdx.x == 0) c->ecg_count = rec + 1;
}

}  // namespace ecg
}  // namespace mb

extern "C" int mbk_ecg(const mb_stencil_dev *st, const double *v, const mb_ecg_dev *e, mb_ctrl *ctrl, cudaStream_t s) {
    mb::ecg::k_ecg_partials<<<MB_ECG_BLOCKS, mb::ecg::NT, 0, s>>>(*st, v, *e, ctrl);
    mb::ecg::k_ecg_finish<<<1, 32, 0, s>>>(*e, ctrl, MB_ECG_BLOCKS);
    return (int)cudaGetLastError();
}

// Resident persistent Jacobi-PCG for the mixed-precision solve on the
// constant-coefficient 7-point operator (kind 0: homogeneous conductivity or a
// diagonal uniform tensor, removed cells by code bytes).  Same Krylov
// recurrences, refinement rule and stopping test as the flat kernel
// (cg_flat.cu), which follow cpu_conjugate_gradient
// (src/linear_system_solver_library/linear_system_solver.c:47-183).
//
// The flat kernel streams its vectors through L2 in every pass (about 29 B per
// cell and pass on the 2 M-cell slab) and its passes wait on that traffic.
// Here each block owns one tile column of the grid (an x-y tile, every z
// plane) and keeps its part of the Krylov iteration on chip for the launch:
//   p (FP32) in shared memory, in a box padded by one cell on every side
//     whose x-y ring holds the neighbouring tiles' values (the halo);
//   A p (FP32) and the correction d = x - x_ref (FP32) in shared memory;
//   r (FP32) and the cells' code bytes in registers.
// x itself stays in global memory as x_ref (FP64), with the FP64 true
// residual r_true = b - A x_ref beside it.  A refinement evaluates
// r_true - A d in FP64 (d at the halo from the owners' boundary copies),
// then folds d into x_ref and r_true; the stopping test uses that FP64
// residual, as in the flat kernel.  The first residual of a launch copies x
// into shared memory (tile, ring and padding) and forms b - A x there.
//
// Only the tile boundary crosses L2 during the iteration: after each U pass
// the owner stores z and d at its boundary cells; in the next Q pass every
// block copies z at its halo (cp.async) and advances the halo's p with the
// same p = z + beta p as the owner applies to the cell, so both copies hold
// the same bits without p itself being exchanged.  The stores happen before
// the block's arrival at the grid reduction (release) and the copies after
// the reduction completes (acquire), so the exchange needs no barrier of its
// own.
//
// The per-row work is branch-free: rows outside the tile, lanes past its
// width and removed cells carry code 0 and their stores are predicated off;
// each row's shared-memory offsets come from a per-block row table, and the
// p box has a fixed row stride, so neighbours in x and y are constant
// offsets.  Loads are issued a batch of rows at a time, ahead of the batch's
// stores.  Per-thread
// partial sums of the FP32 dot products are accumulated in FP32 over the
// thread's cells and added in FP64 across threads and blocks.
//
// Threads: NT per block, one warp per x-row of the tile (lane = x in the
// tile, tiles at most 32 cells wide), rows (k, jy) dealt to the warps
// round-robin, at most RPW rows per warp; one block per SM.
#include "cg_common.cuh"

namespace mb {
namespace rcg {

using fcg::ACTIVE;
using fcg::Args;
using fcg::grid_reduce;

constexpr int BATCH = 4;   // rows whose loads are issued together
constexpr int PW = 34;     // row stride of the p box: 32 cells and the ring

// Tile layout, the same for every block: nbx x nby tiles of tw x th cells
// (the last tile of a row or column may be smaller), each with all nz planes.
struct Tiles {
    int nbx, nby, tw, th;
};

// q = h / d, rem = h - q d for 0 <= h < 2^24, with a float reciprocal of d and
// one correction step (the float estimate is off by less than one)
__device__ __forceinline__ int divmod(int h, int d, float inv_d, int &rem) {
    int q = (int)((float)h * inv_d);
    int r = h - q * d;
    if (r < 0) { q -= 1; r += d; }
    else if (r >= d) { q += 1; r -= d; }
    rem = r;
    return q;
}

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(src) : "memory");
}
// 8 bytes, or zeros when n == 0 (src must still be a valid address)
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int n) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared memory of a tile: the row table, then d and A p (own cells; the A p
// region also stages the halo's z) and the padded p box, or the FP64 copy of
// x over the padded box for the first residual if larger.
__host__ __device__ inline size_t tile_table_bytes(int nt, int rpw) { return (size_t)16 * (nt / 32) * rpw; }
__host__ __device__ inline size_t tile_ap_cells(int tw, int th, int nz) {
    const size_t own = (size_t)tw * th * nz, halo = (size_t)2 * (tw + th) * nz;
    return own > halo ? own : halo;
}
__host__ __device__ inline size_t tile_smem(int tw, int th, int nz, int nt, int rpw) {
    const size_t own = (size_t)tw * th * nz, box = (size_t)PW * (th + 2) * (nz + 2);
    const size_t iter = 4 * (own + tile_ap_cells(tw, th, nz) + box), first = 8 * box;
    return tile_table_bytes(nt, rpw) + (iter > first ? iter : first);
}

template <int NT, int RPW, int HPT>
__global__ void __launch_bounds__(NT, 1) k_rcg(Args a, Tiles T, double *rtrue) {
    constexpr int WARPS = NT / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float inv_tab[64];

    const mb_stencil_dev &st = a.st;
    mb_ctrl *c = a.ctrl;
    const bool pre = c->use_precond != 0;

    const int nx = st.nx, ny = st.ny, nz = st.nz;
    const int bx = (int)blockIdx.x % T.nbx, by = (int)blockIdx.x / T.nbx;
    const int x0 = bx * T.tw, y0 = by * T.th;
    const int tw = min(T.tw, nx - x0), th = min(T.th, ny - y0);
    const bool hw = x0 > 0, he = x0 + tw < nx, hs = y0 > 0, hn = y0 + th < ny;
    const int OW = T.tw, ON = T.tw * T.th * nz;           // own layout [k][jy][ix]
    const int PP = PW * (T.th + 2);                        // box [k+1][jy+1][ix+1]
    const int NB = PP * (nz + 2);
    int4 *rowtab = reinterpret_cast<int4 *>(smem);
    unsigned char *region = smem + tile_table_bytes(NT, RPW);
    float *D = reinterpret_cast<float *>(region);
    float *AP = D + ON;
    float *HZ = AP;                                        // halo z staging (Q pass)
    float *P = AP + tile_ap_cells(T.tw, T.th, nz);
    double *XS = reinterpret_cast<double *>(region);       // first residual only

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lc = min(lane, tw - 1);                      // lanes past the tile repeat its last cell
    const bool edge = (hw && lane == 0) || (he && lane == tw - 1);

    const float a32 = (float)st.alpha, cx = (float)st.cx, cy = (float)st.cy, cz = (float)st.cz;
    double *__restrict__ xg = a.x;
    float *__restrict__ zb = a.z32;    // z at boundary cells
    float *__restrict__ db = a.pa32;   // d at boundary cells

    // Jacobi 1/diag by code byte: alpha plus the coupled faces in the order
    // -x, +x, -y, +y, -z, +z, as k_inv_diag forms it for the flat kernel
    if (threadIdx.x < 64) {
        const unsigned m = threadIdx.x;
        float f = a32;
        const float cf[6] = {cx, cx, cy, cy, cz, cz};
        for (int q = 0; q < 6; ++q)
            if ((m >> q) & 1u) f += cf[q];
        inv_tab[m] = 1.0f / f;
    }
    // row table: p-box index, own index and global index of each row's first
    // cell, boundary flags (1: south side of the tile, 2: north); rows outside
    // the tile point at row (0, 0)
    for (int rho = threadIdx.x; rho < WARPS * RPW; rho += NT) {
        int k = rho / T.th, j = rho - k * T.th;
        const bool ok = k < nz && j < th;
        if (!ok) k = j = 0;
        int4 e;
        e.x = (k + 1) * PP + (j + 1) * PW + 1;
        e.y = (k * T.th + j) * OW;
        e.z = (k * ny + y0 + j) * nx + x0;
        e.w = ok ? ((hs && j == 0) ? 1 : 0) | ((hn && j == th - 1) ? 2 : 0) : 0;
        rowtab[rho] = e;
    }
    // code bytes of this thread's rows (0 outside the tile)
    uint32_t cw[(RPW + 3) / 4];
#pragma unroll
    for (int q = 0; q < (RPW + 3) / 4; ++q) cw[q] = 0u;
#pragma unroll
    for (int s = 0; s < RPW; ++s) {
        const int rho = warp + WARPS * s, k = rho / T.th, j = rho - k * T.th;
        if (k < nz && j < th && lane < tw)
            cw[s >> 2] |= (uint32_t)__ldg(st.code + (size_t)(k * ny + y0 + j) * nx + x0 + lane) << (8 * (s & 3));
    }

    float r[RPW];
#pragma unroll
    for (int s = 0; s < RPW; ++s) r[s] = 0.0f;

    // a pass's view of the code words: an opaque copy, so that the compiler
    // re-extracts the codes in every pass instead of keeping them all live
    uint32_t cv[(RPW + 3) / 4] = {};
    auto fresh_codes = [&]() {
#pragma unroll
        for (int q = 0; q < (RPW + 3) / 4; ++q) asm volatile("mov.b32 %0, %1;" : "=r"(cv[q]) : "r"(cw[q]));
    };
    auto code_of = [&](int s) -> unsigned { return (cv[s >> 2] >> (8 * (s & 3))) & 0xffu; };
    auto row = [&](int s) -> int4 { return rowtab[warp + WARPS * s]; };

    // Halo cells: the four sides' columns/rows of the ring that face another
    // tile, numbered west, east, south, north.
    const int hcol = nz * th, hrow = nz * tw;
    const int nwest = hw ? hcol : 0, neast = he ? hcol : 0, nsouth = hs ? hrow : 0, nnorth = hn ? hrow : 0;
    const int nhalo = nwest + neast + nsouth + nnorth;
    const float inv_th = 1.0f / (float)th, inv_tw = 1.0f / (float)tw;
    auto halo_cell = [&](int h, int &lp) -> size_t {
        int k, rem;
        if (h < nwest + neast) {
            const bool east = h >= nwest;
            k = divmod(east ? h - nwest : h, th, inv_th, rem);
            const int ix = east ? tw : -1;
            lp = (k + 1) * PP + (rem + 1) * PW + ix + 1;
            return ((size_t)k * ny + y0 + rem) * nx + x0 + ix;
        }
        h -= nwest + neast;
        const bool north = h >= nsouth;
        k = divmod(north ? h - nsouth : h, tw, inv_tw, rem);
        const int jy = north ? th : -1;
        lp = (k + 1) * PP + (jy + 1) * PW + rem + 1;
        return ((size_t)k * ny + y0 + jy) * nx + x0 + rem;
    };

    // ---- first residual: x over the padded box into shared memory (FP64,
    // zeros outside the domain), r_true = b - A x, r = (float) r_true, z at
    // the boundary
    for (int i = threadIdx.x; i < NB; i += NT) {
        const int kk = i / PP, rem = i - kk * PP, jj = rem / PW, ii = rem - jj * PW;
        const int gx = x0 + ii - 1, gy = y0 + jj - 1, gz = kk - 1;
        const bool in = ii <= tw + 1 && jj <= th + 1 && gx >= 0 && gx < nx && gy >= 0 && gy < ny && gz >= 0 && gz < nz;
        cp_async8(&XS[i], in ? xg + ((size_t)gz * ny + gy) * nx + gx : xg, in ? 8 : 0);
    }
    cp_async_wait_all();
    __syncthreads();
    int red = 0;
    double rz, rr, error, rr_ref;
    {
        double acc[3] = {0.0, 0.0, 0.0}, s3[3];
        const double a64 = st.alpha, cx64 = st.cx, cy64 = st.cy, cz64 = st.cz;
        fresh_codes();
#pragma unroll
        for (int s0 = 0; s0 < RPW; s0 += BATCH) {
            double bv[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const size_t g = (size_t)row(s0 + u).z + lc;
                bv[u] = a.b ? a.b[g] : a64 * a.vstar[g];
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int s = s0 + u;
                const int4 e = row(s);
                const unsigned m = code_of(s);
                const bool act = m & ACTIVE;
                const int lp = e.x + lc;
                const double xc = XS[lp];
                double ax = a64 * xc;
                ax += (m & 1u) ? cx64 * (xc - XS[lp - 1]) : 0.0;
                ax += (m & 2u) ? cx64 * (xc - XS[lp + 1]) : 0.0;
                ax += (m & 4u) ? cy64 * (xc - XS[lp - PW]) : 0.0;
                ax += (m & 8u) ? cy64 * (xc - XS[lp + PW]) : 0.0;
                ax += (m & 16u) ? cz64 * (xc - XS[lp - PP]) : 0.0;
                ax += (m & 32u) ? cz64 * (xc - XS[lp + PP]) : 0.0;
                const double r64 = act ? bv[u] - ax : 0.0;
                const size_t g = (size_t)e.z + lc;
                if (act) rtrue[g] = r64;
                const float rt = (float)r64;
                const float z = pre ? inv_tab[m & 63u] * rt : rt;
                r[s] = rt;
                acc[0] += (double)rt * (double)z;
                acc[1] += (double)rt * (double)rt;
                acc[2] += r64 * r64;
                if (act && (edge || e.w)) zb[g] = z;
            }
        }
        if (!grid_reduce<3, NT>(a, acc, s3, red)) return;
        rz = s3[0];
        rr = s3[1];
        error = s3[2];
        rr_ref = s3[2];
    }
    // d = 0, p = 0 (box, ring and padding) for the iteration
    for (int i = threadIdx.x; i < ON; i += NT) D[i] = 0.0f;
    for (int i = threadIdx.x; i < NB; i += NT) P[i] = 0.0f;
    __syncthreads();

    const double tol = c->tol;
    const int max_its = c->max_its;
    const double ratio = c->refine_ratio;
    int its = 1, refinements = 1;
    bool done = !(error >= tol) || !(1 < max_its);
    bool first = true;
    double beta = 0.0;

    while (!done) {
        // ---- Q: p = z + beta p (p = z after a restart) on the cells and the
        // halo, then A p and the partial sum of p.Ap
        const float bt = (float)beta;
        int hl[HPT];
#pragma unroll
        for (int q = 0; q < HPT; ++q) {
            const int h = threadIdx.x + q * NT;
            hl[q] = -1;
            if (h < nhalo) cp_async4(&HZ[h], zb + halo_cell(h, hl[q]));
        }
        fresh_codes();
#pragma unroll
        for (int s0 = 0; s0 < RPW; s0 += BATCH) {
            int lp[BATCH];
            float po[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                lp[u] = row(s0 + u).x + lc;
                po[u] = P[lp[u]];
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const unsigned m = code_of(s0 + u);
                const float z = pre ? inv_tab[m & 63u] * r[s0 + u] : r[s0 + u];
                const float pn = first ? z : __fmaf_rn(bt, po[u], z);
                if (m & ACTIVE) P[lp[u]] = pn;
            }
        }
        cp_async_wait_all();
#pragma unroll
        for (int q = 0; q < HPT; ++q) {
            if (hl[q] >= 0) {
                const float zh = HZ[threadIdx.x + q * NT];
                P[hl[q]] = first ? zh : __fmaf_rn(bt, P[hl[q]], zh);
            }
        }
        __syncthreads();
        float q1f = 0.0f;
        fresh_codes();
#pragma unroll
        for (int s0 = 0; s0 < RPW; s0 += BATCH) {
            float pv[BATCH][7];
            int la[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int4 e = row(s0 + u);
                const float *pp = P + e.x + lc;
                la[u] = e.y + lc;
                pv[u][0] = pp[0];
                pv[u][1] = pp[-1];
                pv[u][2] = pp[1];
                pv[u][3] = pp[-PW];
                pv[u][4] = pp[PW];
                pv[u][5] = pp[-PP];
                pv[u][6] = pp[PP];
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const unsigned m = code_of(s0 + u);
                const float pc = pv[u][0];
                float v = a32 * pc;
                v += (m & 1u) ? cx * (pc - pv[u][1]) : 0.0f;
                v += (m & 2u) ? cx * (pc - pv[u][2]) : 0.0f;
                v += (m & 4u) ? cy * (pc - pv[u][3]) : 0.0f;
                v += (m & 8u) ? cy * (pc - pv[u][4]) : 0.0f;
                v += (m & 16u) ? cz * (pc - pv[u][5]) : 0.0f;
                v += (m & 32u) ? cz * (pc - pv[u][6]) : 0.0f;
                const bool act = m & ACTIVE;
                if (act) AP[la[u]] = v;
                q1f = act ? __fmaf_rn(pc, v, q1f) : q1f;
            }
        }
        double q1[1] = {(double)q1f}, s1[1];
        if (!grid_reduce<1, NT>(a, q1, s1, red)) return;
        const double alpha = (pre ? rz : rr) / s1[0];

        // ---- U: d += alpha p, r -= alpha A p, z = r / diag; z and d to the
        // boundary copies; partial sums of r.z and r.r
        const float al = (float)alpha;
        float u0 = 0.0f, u1 = 0.0f;
        fresh_codes();
#pragma unroll
        for (int s0 = 0; s0 < RPW; s0 += BATCH) {
            float pv[BATCH], dv[BATCH], av[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int4 e = row(s0 + u);
                const int l = e.y + lc;
                pv[u] = P[e.x + lc];
                dv[u] = D[l];
                av[u] = AP[l];
            }
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int s = s0 + u;
                const unsigned m = code_of(s);
                const bool act = m & ACTIVE;
                const int4 e = row(s);
                const float dn = __fmaf_rn(al, pv[u], dv[u]);
                const float rn = act ? __fmaf_rn(-al, av[u], r[s]) : 0.0f;
                r[s] = rn;
                if (act) D[e.y + lc] = dn;
                const float z = pre ? inv_tab[m & 63u] * rn : rn;
                u0 = __fmaf_rn(z, rn, u0);
                u1 = __fmaf_rn(rn, rn, u1);
                if (act && (edge || e.w)) {
                    const size_t g = (size_t)e.z + lc;
                    zb[g] = z;
                    db[g] = dn;
                }
            }
        }
        double u2[2] = {(double)u0, (double)u1}, s2[2];
        if (!grid_reduce<2, NT>(a, u2, s2, red)) return;
        its += 1;
        if (s2[1] <= fmax(c->refine_floor, ratio * rr_ref) || its >= max_its) {
            // ---- refinement: r_true -= A d in FP64 (the FP64 residual of
            // x_ref + d), r = (float) r_true, restart from it.  d goes over
            // the padded box (own cells from D, the halo from the owners'
            // boundary copies); p's values there are not needed again.
            fresh_codes();
#pragma unroll
            for (int s = 0; s < RPW; ++s) {
                const int4 e = row(s);
                if (code_of(s) & ACTIVE) P[e.x + lc] = D[e.y + lc];
            }
#pragma unroll
            for (int q = 0; q < HPT; ++q) {
                const int h = threadIdx.x + q * NT;
                if (h < nhalo) {
                    int lp;
                    const size_t g = halo_cell(h, lp);
                    cp_async4(&P[lp], db + g);
                }
            }
            cp_async_wait_all();
            __syncthreads();
            double t3[3] = {0.0, 0.0, 0.0}, s3[3];
            const double a64 = st.alpha, cx64 = st.cx, cy64 = st.cy, cz64 = st.cz;
            fresh_codes();
#pragma unroll
            for (int s0 = 0; s0 < RPW; s0 += BATCH) {
                double rv[BATCH];
#pragma unroll
                for (int u = 0; u < BATCH; ++u) rv[u] = rtrue[(size_t)row(s0 + u).z + lc];
#pragma unroll
                for (int u = 0; u < BATCH; ++u) {
                    const int s = s0 + u;
                    const int4 e = row(s);
                    const unsigned m = code_of(s);
                    const bool act = m & ACTIVE;
                    const int lp = e.x + lc;
                    const double dc = P[lp];
                    double ad = a64 * dc;
                    ad += (m & 1u) ? cx64 * (dc - (double)P[lp - 1]) : 0.0;
                    ad += (m & 2u) ? cx64 * (dc - (double)P[lp + 1]) : 0.0;
                    ad += (m & 4u) ? cy64 * (dc - (double)P[lp - PW]) : 0.0;
                    ad += (m & 8u) ? cy64 * (dc - (double)P[lp + PW]) : 0.0;
                    ad += (m & 16u) ? cz64 * (dc - (double)P[lp - PP]) : 0.0;
                    ad += (m & 32u) ? cz64 * (dc - (double)P[lp + PP]) : 0.0;
                    const double r64 = act ? rv[u] - ad : 0.0;
                    const size_t g = (size_t)e.z + lc;
                    if (act) rtrue[g] = r64;
                    const float rt = (float)r64;
                    const float z = pre ? inv_tab[m & 63u] * rt : rt;
                    r[s] = rt;
                    t3[0] += (double)rt * (double)z;
                    t3[1] += (double)rt * (double)rt;
                    t3[2] += r64 * r64;
                    if (act && (edge || e.w)) zb[g] = z;
                }
            }
            if (!grid_reduce<3, NT>(a, t3, s3, red)) return;
            // fold d into x_ref (every reader of d in this block has passed
            // the reduction; other blocks read only the boundary copies)
            fresh_codes();
#pragma unroll
            for (int s0 = 0; s0 < RPW; s0 += BATCH) {
                double xv[BATCH];
#pragma unroll
                for (int u = 0; u < BATCH; ++u) xv[u] = xg[(size_t)row(s0 + u).z + lc];
#pragma unroll
                for (int u = 0; u < BATCH; ++u) {
                    const int s = s0 + u;
                    if (code_of(s) & ACTIVE) {
                        const int4 e = row(s);
                        xg[(size_t)e.z + lc] = xv[u] + (double)D[e.y + lc];
                        D[e.y + lc] = 0.0f;
                    }
                }
            }
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
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->its = its;
        c->error = error;
        c->refinements = refinements;
        c->rz = rz;
        c->rr = rr;
        c->done = 1;
    }
}

// (threads, rows per warp, halo cells per thread) shapes, smallest first
struct Shape {
    int nt, rpw, hpt;
    const void *fn;
};
#define MB_SHAPE(N, R, H) {N, R, H, (const void *)k_rcg<N, R, H>}
static const Shape kShapes[] = {
    MB_SHAPE(512, 4, 2), MB_SHAPE(512, 8, 4), MB_SHAPE(512, 16, 4), MB_SHAPE(512, 16, 8), MB_SHAPE(512, 32, 8),
    MB_SHAPE(512, 32, 16),
};
#undef MB_SHAPE
constexpr int NUM_SHAPES = sizeof(kShapes) / sizeof(kShapes[0]);

}  // namespace rcg
}  // namespace mb

using namespace mb::rcg;

// Lays the grid out in tile columns for the resident kernel and checks that
// they fit: at most one block per SM, tiles at most 32 cells wide, every row
// of a tile within the rows of its warps, the tile within the shared memory a
// block may opt in to, cell indices within 32 bits.  Fills the plan fields
// of *p and returns 1, or returns 0 when the kernel does not apply (FP64, a
// non-constant operator, or a tile that does not fit).
extern "C" int mbk_rcg_plan(mb_pcg_dev *p) {
    if (!p->mixed || p->st.kind != 0 || !p->st.code) return 0;
    int dev = 0, sms = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    const long long nx = p->st.nx, ny = p->st.ny, nz = p->st.nz;
    if (nx < 2 || ny < 1 || nz < 1 || nx * ny * nz >= (1LL << 31)) return 0;
    long long nbx = (nx + 31) / 32;
    const long long tw = (nx + nbx - 1) / nbx;
    nbx = (nx + tw - 1) / tw;
    const long long nby_max = sms / nbx;
    if (nby_max < 1) return 0;
    const long long th = (ny + nby_max - 1) / nby_max;
    const long long nby = (ny + th - 1) / th;
    const long long rows = th * nz, halo = 2 * (tw + th) * nz;
    for (int v = 0; v < NUM_SHAPES; ++v) {
        const Shape &sh = kShapes[v];
        if (rows > (long long)(sh.nt / 32) * sh.rpw || halo > (long long)sh.nt * sh.hpt) continue;
        const size_t dyn = tile_smem((int)tw, (int)th, (int)nz, sh.nt, sh.rpw);
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, sh.fn) != cudaSuccess) return 0;
        if (dyn + fa.sharedSizeBytes > (size_t)optin) return 0;
        if (cudaFuncSetAttribute(sh.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) != cudaSuccess) return 0;
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sh.fn, sh.nt, dyn) != cudaSuccess || per < 1) return 0;
        if (nbx * nby > (long long)sms * per) return 0;
        p->rc_shape = v;
        p->rc_nbx = (int)nbx;
        p->rc_nby = (int)nby;
        p->rc_tw = (int)tw;
        p->rc_th = (int)th;
        p->rc_smem = dyn;
        return 1;
    }
    return 0;
}

extern "C" int mbk_rcg_launch(const mb_pcg_dev *p, cudaStream_t s) {
    if (p->rc_shape < 0 || p->rc_shape >= NUM_SHAPES || !p->rtrue || !p->pa32 || !p->z32)
        return (int)cudaErrorInvalidValue;
    Args a;
    a.st = p->st;
    a.x = p->x; a.vstar = p->vstar; a.b = p->b;
    a.r64 = p->r64; a.pa64 = p->pa64; a.pb64 = p->pb64; a.z64 = p->z64;
    a.r32 = p->r32; a.pa32 = p->pa32; a.pb32 = p->pb32; a.z32 = p->z32;
    a.inv_diag64 = p->inv_diag64; a.inv_diag32 = p->inv_diag32;
    a.partials = p->partials; a.ctrl = p->ctrl; a.bar = p->bar; a.status = p->status;
    Tiles t{p->rc_nbx, p->rc_nby, p->rc_tw, p->rc_th};
    double *rtrue = p->rtrue;
    // the arrival counter starts from zero in every launch
    cudaError_t e = cudaMemsetAsync(p->bar, 0, 2 * sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    void *args[] = {&a, &t, &rtrue};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(p->rc_nbx * p->rc_nby));
    cfg.blockDim = dim3((unsigned)kShapes[p->rc_shape].nt);
    cfg.dynamicSmemBytes = p->rc_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelExC(&cfg, kShapes[p->rc_shape].fn, args);
}

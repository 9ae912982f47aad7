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
//   U: x += alpha p, r -= alpha A p (A p as Q stored it), z = r / diag and
//      the partial sums of r.z and r.r; a streaming pass over the cells' own
//      values.
// p is double-buffered so Q reads p_old of neighbours while writing p_new.
//
// Rows are read without per-cell index arithmetic: each cell carries a code
// byte (which of its six faces couple, and whether it is active; kind 2 a row
// id into the per-plane class table), neighbour indices are the cell's index
// plus fixed strides, clamped into the grid, and each block sweeps a
// contiguous range of cells.
//
// Mixed precision: p, r, z and A p in FP32, the solution x and every dot
// product in FP64; when the FP32 recurrence residual has dropped by
// refine_ratio (or below tol) the FP64 true residual b - A x replaces r and the
// iteration restarts from it; the stopping test uses that FP64 residual.
//
// Launch shapes are template parameters (threads per block, cells gathered
// per thread before use, resident blocks per SM); the host times the
// variants on the tissue's first solve and keeps the fastest.
#include "cg_common.cuh"

namespace mb {
namespace fcg {

// ---- operator rows ------------------------------------------------------------

// A 7-point row gathered for one cell: the field at the cell and at the six
// neighbours (-x, +x, -y, +y, -z, +z), the code byte, and for kind 1 the six
// face coefficients.  Neighbour indices are clamped into the grid, so every
// load of the row is issued at once, independent of the code byte; values
// of faces that do not couple are discarded by row_apply.
template <typename T, int KIND>
struct Row7 {
    T pc, p[6];
    T c[KIND == 1 ? 6 : 1];
    unsigned m;
};

template <typename T, int KIND, typename PF>
__device__ __forceinline__ Row7<T, KIND> gather7(const mb_stencil_dev &st, uint32_t g, PF pf) {
    Row7<T, KIND> R;
    const uint32_t sy = (uint32_t)st.nx, sz = (uint32_t)st.nx * (uint32_t)st.ny, n = sz * (uint32_t)st.nz;
    const uint32_t i0 = g > 0u ? g - 1u : g, i1 = g + 1u < n ? g + 1u : g;
    const uint32_t i2 = g >= sy ? g - sy : g, i3 = g + sy < n ? g + sy : g;
    const uint32_t i4 = g >= sz ? g - sz : g, i5 = g + sz < n ? g + sz : g;
    R.m = __ldg(st.code + g);
    R.pc = pf(g);
    R.p[0] = pf(i0);
    R.p[1] = pf(i1);
    R.p[2] = pf(i2);
    R.p[3] = pf(i3);
    R.p[4] = pf(i4);
    R.p[5] = pf(i5);
    if constexpr (KIND == 1) {
        R.c[0] = T(__ldg(st.fx + i0));
        R.c[1] = T(__ldg(st.fx + g));
        R.c[2] = T(__ldg(st.fy + i2));
        R.c[3] = T(__ldg(st.fy + g));
        R.c[4] = T(__ldg(st.fz + i4));
        R.c[5] = T(__ldg(st.fz + g));
    }
    return R;
}

// (A p)_c = alpha p_c + sum over coupled faces of c (p_c - p_n).
template <typename T, int KIND>
__device__ __forceinline__ T row_apply(const mb_stencil_dev &st, const Row7<T, KIND> &R) {
    T acc = T(st.alpha) * R.pc;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        T c;
        if constexpr (KIND == 0) c = T(q < 2 ? st.cx : (q < 4 ? st.cy : st.cz));
        else c = R.c[q];
        if ((R.m >> q) & 1u) acc += c * (R.pc - R.p[q]);
    }
    return acc;
}

// 27-point rows (kind 2) from the per-plane class table; the product is
// formed while gathering.  Missing neighbours have zero coefficients in the
// table and are not loaded; entries that are zero in every row of the table
// (st.nzmask) are not read at all.
template <typename T>
struct Row27 {
    T pc, ap;
    unsigned m;
};

template <typename T, typename PF>
__device__ __forceinline__ Row27<T> gather27(const mb_stencil_dev &st, uint32_t g, PF pf) {
    Row27<T> R;
    R.m = ACTIVE;
    R.pc = pf(g);
    const int sy = st.nx, sz = st.nx * st.ny;
    const size_t row = (size_t)__ldg(st.rowid + g) * 27;
    T acc = T(0);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const int q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                if (!((st.nzmask >> q) & 1u)) continue;     // zero in every row
                const T c = sizeof(T) == 8 ? T(__ldg(st.table + row + q)) : T(__ldg(st.table32 + row + q));
                if (q == 13) acc += c * R.pc;
                else if (c != T(0)) acc += c * pf((uint32_t)((int)g + dx + sy * dy + sz * dz));
            }
    R.ap = acc;
    return R;
}

template <typename T, int KIND, typename PF>
__device__ __forceinline__ auto gather(const mb_stencil_dev &st, uint32_t g, PF pf) {
    if constexpr (KIND == 2) return gather27<T>(st, g, pf);
    else return gather7<T, KIND>(st, g, pf);
}

template <typename T, int KIND, typename R>
__device__ __forceinline__ T product(const mb_stencil_dev &st, const R &row) {
    if constexpr (KIND == 2) return row.ap;
    else return row_apply<T, KIND>(st, row);
}

// ---- sweeps ------------------------------------------------------------------

// Contiguous, warp-aligned range of cells owned by this block.
__device__ __forceinline__ void block_chunk(uint32_t n, uint32_t &c0, uint32_t &c1) {
    const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 31u) & ~31u;
    c0 = min(n, blockIdx.x * chunk);
    c1 = min(n, c0 + chunk);
}

// The units (cells or groups) a thread visits in a pass, in rounds of
// per_round = U x blockDim units per block: unit base + u blockDim (u < U) for
// base = start, start + step, ... below end.
//   ORD 0: each block sweeps its own contiguous range (block_chunk).
//   ORD 1: interleaved -- round r of block b covers units
//          [(r G + b) per_round, (r G + b + 1) per_round), G blocks, so the
//          whole grid moves through the cells together and the rows a round
//          reads one z-plane away were read a few rounds before (still in
//          L2 when a pass streams far more than L2 holds).
template <int ORD>
struct Sweep {
    uint32_t start, end, step;
    __device__ __forceinline__ Sweep(uint32_t units, uint32_t per_round) {
        if constexpr (ORD == 0) {
            uint32_t c0, c1;
            block_chunk(units, c0, c1);
            start = c0 + threadIdx.x;
            end = c1;
            step = per_round;
        } else {
            start = blockIdx.x * per_round + threadIdx.x;
            end = units;
            step = gridDim.x * per_round;
        }
    }
};

// A pass over the active cells: each thread takes U cells of the block's range
// at a time and gathers all U rows (their loads in flight together) before
// using them.
template <typename T, int KIND, int NT, int U, int ORD, typename PF, typename ACT>
__device__ __forceinline__ void pass(const mb_stencil_dev &st, PF pf, ACT act) {
    const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
    const uint32_t nt = blockDim.x;     // <= NT: the host sizes blocks to whole rounds
    const Sweep<ORD> sw(n, U * nt);
    for (uint32_t base = sw.start; base < sw.end; base += sw.step) {
        decltype(gather<T, KIND>(st, 0u, pf)) rows[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t g = base + u * nt;
            rows[u] = gather<T, KIND>(st, g < sw.end ? g : base, pf);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t g = base + u * nt;
            if (g < sw.end && (rows[u].m & ACTIVE)) act(g, rows[u]);
        }
    }
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

// Jacobi 1/diag of a cell: with constant coefficients (kind 0) it depends on
// the code byte only and comes from the block's 64-entry table (filled by
// fill_inv_table as k_inv_diag forms it), otherwise from the per-cell array.
template <bool MIXED, int KIND>
__device__ __forceinline__ typename Prec<MIXED>::T inv_of(const Args &a, const typename Prec<MIXED>::T *tab,
                                                         uint32_t g, unsigned m) {
    if constexpr (KIND == 0) return tab[m & 63u];
    else return inv_d<MIXED>(a, g);
}

// Fills the block's table; a block may have as few as 32 threads (the host
// sizes blocks to whole rounds of cells).
template <bool MIXED>
__device__ __forceinline__ void fill_inv_table(const mb_stencil_dev &st, typename Prec<MIXED>::T *tab) {
    for (unsigned m = threadIdx.x; m < 64; m += blockDim.x) {
        const double c[6] = {st.cx, st.cx, st.cy, st.cy, st.cz, st.cz};
        double d64 = st.alpha;
        float d32 = (float)st.alpha;
        for (int q = 0; q < 6; ++q)
            if ((m >> q) & 1u) {
                d64 += c[q];
                d32 += (float)c[q];
            }
        if constexpr (MIXED) tab[m] = 1.0f / d32;
        else tab[m] = 1.0 / d64;
    }
}

// ---- four cells per thread ----------------------------------------------------
//
// With nx a multiple of 4, a thread takes 4 consecutive cells of an x-row
// (a group, first index g0 a multiple of 4) and reads every row of the
// stencil as one 16-byte load (two for doubles): the group itself, the rows
// at -y, +y, -z, +z (kind 2: the nine rows dy, dz in -1..1), plus one scalar
// on each side for the x neighbours of the group's end cells.  Row indices
// are clamped into the grid; values of neighbours that do not couple are
// discarded (kinds 0, 1) or multiplied by the zero coefficients the class
// table holds for them (kind 2; rows and entries that are zero in every row
// of the table are skipped).  Sums run in the same order as the
// one-cell-per-thread rows above, so both forms give the same values.

template <typename T>
struct Vec4 { T v[4]; };

__device__ __forceinline__ Vec4<float> ld4(const float *p, uint32_t i) {
    const float4 f = *reinterpret_cast<const float4 *>(p + i);
    return {{f.x, f.y, f.z, f.w}};
}
__device__ __forceinline__ Vec4<double> ld4(const double *p, uint32_t i) {
    const double2 a = *reinterpret_cast<const double2 *>(p + i);
    const double2 b = *reinterpret_cast<const double2 *>(p + i + 2);
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float *p, uint32_t i, const Vec4<float> &v) {
    *reinterpret_cast<float4 *>(p + i) = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
__device__ __forceinline__ void st4(double *p, uint32_t i, const Vec4<double> &v) {
    *reinterpret_cast<double2 *>(p + i) = make_double2(v.v[0], v.v[1]);
    *reinterpret_cast<double2 *>(p + i + 2) = make_double2(v.v[2], v.v[3]);
}

// Field readers: row(i) = the 4 values at i..i+3 (i a multiple of 4), at(i) =
// one value.
template <typename T>
struct Plain {
    const T *f;
    __device__ __forceinline__ Vec4<T> row(uint32_t i) const { return ld4(f, i); }
    __device__ __forceinline__ T at(uint32_t i) const { return f[i]; }
};
// p_new = z + beta p_old, formed where it is read.
template <typename T>
struct Direction {
    const T *z, *p;
    T beta;
    __device__ __forceinline__ Vec4<T> row(uint32_t i) const {
        const Vec4<T> a = ld4(z, i), b = ld4(p, i);
        Vec4<T> o;
#pragma unroll
        for (int k = 0; k < 4; ++k) o.v[k] = a.v[k] + beta * b.v[k];
        return o;
    }
    __device__ __forceinline__ T at(uint32_t i) const { return z[i] + beta * p[i]; }
};

// The values left of a stencil row's first cell and right of its last.  The
// lanes of a warp hold consecutive groups, so where the lane below holds the
// group g0 - 4 of the same x-row (lc), its row for the same (dz, dy) starts
// at b - 4 (rows of one x-row are clamped alike) and the value left of this
// row is the last one it read: it comes by shuffle, and likewise from the
// lane above (rc).  Other lanes (lane 0 and 31, groups on an x face, lanes
// past the end of a range) load it, with a load whose condition is known
// before the row's loads.  The same values as loading every one of them,
// without the 16-byte-strided scalar loads.  All 32 lanes call it together.
template <typename T, typename F>
__device__ __forceinline__ void x_sides(const F &f, bool lc, bool rc, uint32_t b, uint32_t n, const Vec4<T> &mid,
                                        bool need_l, bool need_r, T &wl, T &wr) {
    T l = T(0), r = T(0);
    if (need_l && !lc) l = f.at(b > 0 ? b - 1 : b);
    if (need_r && !rc) r = f.at(b + 4 < n ? b + 4 : b);
    const T sl = __shfl_up_sync(0xffffffffu, mid.v[3], 1);
    const T sr = __shfl_down_sync(0xffffffffu, mid.v[0], 1);
    wl = lc ? sl : l;
    wr = rc ? sr : r;
}

// (A f) for the group at g0: pc = f at the 4 cells, ap = the products, m =
// the cells' code bytes (kind 2: all active).  All 32 lanes call it together.
template <typename T, int KIND, typename F>
__device__ __forceinline__ void apply4(const mb_stencil_dev &st, uint32_t g0, const F &f, Vec4<T> &pc, Vec4<T> &ap,
                                       unsigned (&m)[4]) {
    const uint32_t sy = (uint32_t)st.nx, sz = (uint32_t)st.nx * (uint32_t)st.ny, n = sz * (uint32_t)st.nz;
    pc = f.row(g0);
    if constexpr (KIND == 2) {
        const unsigned lane = threadIdx.x & 31u;
        const uint32_t gl = __shfl_up_sync(0xffffffffu, g0, 1), gr = __shfl_down_sync(0xffffffffu, g0, 1);
        // the lane below / above holds the adjacent group of the same x-row
        bool lc = lane != 0u && gl + 4u == g0, rc = lane != 31u && gr == g0 + 4u;
        const ushort4 rid = *reinterpret_cast<const ushort4 *>(st.rowid + g0);
        // x class of the first / last cell (row id = k 9 + y class 3 + x class)
        lc = lc && (rid.x % 3u) != 0u;
        rc = rc && (rid.w % 3u) != 2u;
        const size_t rw[4] = {(size_t)rid.x * 27, (size_t)rid.y * 27, (size_t)rid.z * 27, (size_t)rid.w * 27};
        // away from the x faces the four cells share one table row
        const bool uni = rid.x == rid.y && rid.x == rid.z && rid.x == rid.w;
        T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                // entries dx = -1, 0, +1 of this row that are non-zero
                // somewhere in the table (the same for every thread)
                const unsigned rb = (st.nzmask >> ((dz + 1) * 9 + (dy + 1) * 3)) & 7u;
                if (!rb) continue;
                uint32_t b = g0;
                if (dz < 0) b = b >= sz ? b - sz : g0;
                if (dz > 0) b = b + sz < n ? b + sz : g0;
                if (dy < 0) b = b >= sy ? b - sy : g0;
                if (dy > 0) b = b + sy < n ? b + sy : g0;
                const Vec4<T> mid = (dz == 0 && dy == 0) ? pc : f.row(b);
                T w[6];
                x_sides<T>(f, lc, rc, b, n, mid, (rb & 1u) != 0u, (rb & 4u) != 0u, w[0], w[5]);
#pragma unroll
                for (int k = 0; k < 4; ++k) w[k + 1] = mid.v[k];
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!((rb >> (dx + 1)) & 1u)) continue;
                    const int q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                    const T c0 = sizeof(T) == 8 ? T(__ldg(st.table + rw[0] + q)) : T(__ldg(st.table32 + rw[0] + q));
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        T c = c0;
                        if (k && !uni) c = sizeof(T) == 8 ? T(__ldg(st.table + rw[k] + q)) : T(__ldg(st.table32 + rw[k] + q));
                        acc[k] += c * w[k + 1 + dx];
                    }
                }
            }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            ap.v[k] = acc[k];
            m[k] = ACTIVE;
        }
    } else {
        const uchar4 cd = *reinterpret_cast<const uchar4 *>(st.code + g0);
        m[0] = cd.x; m[1] = cd.y; m[2] = cd.z; m[3] = cd.w;
        // two values per group: plain loads (the shuffles' bookkeeping costs
        // registers these forms do not have to spare)
        const T xl = f.at(g0 > 0 ? g0 - 1 : g0), xr = f.at(g0 + 4 < n ? g0 + 4 : g0);
        const Vec4<T> ym = f.row(g0 >= sy ? g0 - sy : g0), yp = f.row(g0 + sy < n ? g0 + sy : g0);
        const Vec4<T> zm = f.row(g0 >= sz ? g0 - sz : g0), zp = f.row(g0 + sz < n ? g0 + sz : g0);
        T c[6][4];
        if constexpr (KIND == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                c[0][k] = c[1][k] = T(st.cx);
                c[2][k] = c[3][k] = T(st.cy);
                c[4][k] = c[5][k] = T(st.cz);
            }
        } else {
            const Vec4<double> fx = ld4(st.fx, g0), fy = ld4(st.fy, g0), fz = ld4(st.fz, g0);
            const Vec4<double> fym = ld4(st.fy, g0 >= sy ? g0 - sy : g0), fzm = ld4(st.fz, g0 >= sz ? g0 - sz : g0);
            const double fxl = __ldg(st.fx + (g0 > 0 ? g0 - 1 : g0));
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                c[0][k] = T(k ? fx.v[k - 1] : fxl);
                c[1][k] = T(fx.v[k]);
                c[2][k] = T(fym.v[k]);
                c[3][k] = T(fy.v[k]);
                c[4][k] = T(fzm.v[k]);
                c[5][k] = T(fz.v[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const T p = pc.v[k];
            const T nb[6] = {k ? pc.v[k - 1] : xl, k < 3 ? pc.v[k + 1] : xr, ym.v[k], yp.v[k], zm.v[k], zp.v[k]};
            T acc = T(st.alpha) * p;
#pragma unroll
            for (int q = 0; q < 6; ++q)
                if ((m[k] >> q) & 1u) acc += c[q][k] * (p - nb[q]);
            ap.v[k] = acc;
        }
    }
}

// A pass over the groups of the block's range: each thread takes U groups at
// a time and forms all U products (their loads in flight together) before
// act(g0, pc, ap, m) runs for each.
template <typename T, int KIND, int NT, int U, int ORD, typename F, typename ACT>
__device__ __forceinline__ void pass4(const mb_stencil_dev &st, const F &f, ACT act) {
    const uint32_t groups = ((uint32_t)st.nx * st.ny * st.nz) >> 2;
    const uint32_t nt = blockDim.x;     // <= NT, a multiple of 32: the host sizes blocks to whole rounds
    const uint32_t lane = threadIdx.x & 31u;
    const Sweep<ORD> sw(groups, U * nt);
    // a warp runs its rounds together (while its first lane's unit is in
    // range; lanes past the end repeat the range's last group and skip act),
    // as apply4's shuffles need
    for (uint32_t q = sw.start; q - lane < sw.end; q += sw.step) {
        Vec4<T> pc[U], ap[U];
        unsigned m[U][4];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t qq = q + u * nt;
            apply4<T, KIND>(st, (qq < sw.end ? qq : sw.end - 1u) << 2, f, pc[u], ap[u], m[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (q + u * nt < sw.end) act((q + u * nt) << 2, pc[u], ap[u], m[u]);
    }
}

// ---- the three passes, for either layout ---------------------------------------

// FP64 true residual r = b - A x; stores r (in T), z and p = z; accumulates
// r.z (T products, FP64 sums), r.r of the stored r, and the FP64 r.r.
template <bool MIXED, int KIND, int NT, int U, bool VEC, int ORD>
__device__ __forceinline__ void residual_pass(const Args &a, typename Prec<MIXED>::T *r,
                                              typename Prec<MIXED>::T *p, bool pre,
                                              const typename Prec<MIXED>::T *itab, double (&acc)[3]) {
    using T = typename Prec<MIXED>::T;
    const mb_stencil_dev &st = a.st;
    const double *__restrict__ x = a.x;
    if constexpr (VEC) {
        pass4<double, KIND, NT, U, ORD>(st, Plain<double>{x}, [&](uint32_t g0, const Vec4<double> &xc, const Vec4<double> &ax,
                                                        const unsigned (&m)[4]) {
            Vec4<T> rv = ld4(r, g0), pv = ld4(p, g0);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!(m[k] & ACTIVE)) continue;
                const uint32_t g = g0 + k;
                const double bb = a.b ? a.b[g] : st.alpha * a.vstar[g];
                const double r64 = bb - ax.v[k];
                const T rt = (T)r64;
                const T z = pre ? inv_of<MIXED, KIND>(a, itab, g, m[k]) * rt : rt;
                rv.v[k] = rt;
                pv.v[k] = z;
                acc[0] += (double)rt * (double)z;
                acc[1] += (double)rt * (double)rt;
                acc[2] += r64 * r64;
            }
            st4(r, g0, rv);
            st4(p, g0, pv);
        });
    } else {
        pass<double, KIND, NT, U, ORD>(st, [&](uint32_t q) { return x[q]; },
                                  [&](uint32_t g, const auto &row) {
                                      const double ax = product<double, KIND>(st, row);
                                      const double bb = a.b ? a.b[g] : st.alpha * a.vstar[g];
                                      const double r64 = bb - ax;
                                      const T rt = (T)r64;
                                      const T z = pre ? inv_of<MIXED, KIND>(a, itab, g, row.m) * rt : rt;
                                      r[g] = rt;
                                      p[g] = z;
                                      acc[0] += (double)rt * (double)z;
                                      acc[1] += (double)rt * (double)rt;
                                      acc[2] += r64 * r64;
                                  });
    }
}

// Q: the direction (p_new = z + beta p_old, or p itself on a restart), stored
// when new, A p stored for the U pass, and the partial sum of p.Ap.
template <bool MIXED, int KIND, int NT, int U, bool VEC, int ORD>
__device__ __forceinline__ void q_pass(const Args &a, bool first, const typename Prec<MIXED>::T *po,
                                       typename Prec<MIXED>::T *pw, const typename Prec<MIXED>::T *zb,
                                       typename Prec<MIXED>::T *apb, double beta, double &q1) {
    using T = typename Prec<MIXED>::T;
    const mb_stencil_dev &st = a.st;
    const T bt = (T)beta;
    if constexpr (VEC) {
        auto dot = [&](const Vec4<T> &pc, const Vec4<T> &ap, const unsigned (&m)[4]) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (m[k] & ACTIVE) q1 += (double)pc.v[k] * (double)ap.v[k];
        };
        if (first) {
            pass4<T, KIND, NT, U, ORD>(st, Plain<T>{po}, [&](uint32_t g0, const Vec4<T> &pc, const Vec4<T> &ap,
                                                     const unsigned (&m)[4]) {
                st4(apb, g0, ap);
                dot(pc, ap, m);
            });
        } else {
            pass4<T, KIND, NT, U, ORD>(st, Direction<T>{zb, po, bt}, [&](uint32_t g0, const Vec4<T> &pc, const Vec4<T> &ap,
                                                                 const unsigned (&m)[4]) {
                st4(pw, g0, pc);
                st4(apb, g0, ap);
                dot(pc, ap, m);
            });
        }
    } else {
        if (first) {
            pass<T, KIND, NT, U, ORD>(st, [&](uint32_t q) { return po[q]; },
                                 [&](uint32_t g, const auto &row) {
                                     const T ap = product<T, KIND>(st, row);
                                     apb[g] = ap;
                                     q1 += (double)row.pc * (double)ap;
                                 });
        } else {
            pass<T, KIND, NT, U, ORD>(st, [&](uint32_t q) { return zb[q] + bt * po[q]; },
                                 [&](uint32_t g, const auto &row) {
                                     pw[g] = row.pc;
                                     const T ap = product<T, KIND>(st, row);
                                     apb[g] = ap;
                                     q1 += (double)row.pc * (double)ap;
                                 });
        }
    }
}

// U: x += alpha p, r -= alpha A p (A p as the Q pass stored it), z = r / diag;
// partial sums of r.z and r.r.  A streaming pass: every value it reads is the
// cell's own.  z of removed cells is stored as 0 (no active cell couples to
// them).
template <bool MIXED, int KIND, int NT, int U, bool VEC, int ORD>
__device__ __forceinline__ void u_pass(const Args &a, const typename Prec<MIXED>::T *pc_,
                                       const typename Prec<MIXED>::T *apb, typename Prec<MIXED>::T *r,
                                       typename Prec<MIXED>::T *zb, bool pre, const typename Prec<MIXED>::T *itab,
                                       double alpha, double (&u2)[2]) {
    using T = typename Prec<MIXED>::T;
    const mb_stencil_dev &st = a.st;
    const T al = (T)alpha;
    double *__restrict__ x = a.x;
    const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
    const uint32_t nt = blockDim.x;
    if constexpr (VEC) {
        const Sweep<ORD> sw(n >> 2, U * nt);
        for (uint32_t q = sw.start; q < sw.end; q += sw.step) {
            Vec4<T> pv[U], av[U], rv[U], id[U];
            Vec4<double> xv[U];
            unsigned m[U][4];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t qq = q + u * nt;
                const uint32_t g0 = (qq < sw.end ? qq : q) << 2;
                if constexpr (KIND == 2) {
                    m[u][0] = m[u][1] = m[u][2] = m[u][3] = ACTIVE;
                } else {
                    const uchar4 cd = *reinterpret_cast<const uchar4 *>(st.code + g0);
                    m[u][0] = cd.x; m[u][1] = cd.y; m[u][2] = cd.z; m[u][3] = cd.w;
                }
                pv[u] = ld4(pc_, g0);
                av[u] = ld4(apb, g0);
                rv[u] = ld4(r, g0);
                xv[u] = ld4(x, g0);
                if constexpr (KIND != 0) {
                    if (pre) {
                        if constexpr (MIXED) id[u] = ld4(a.inv_diag32, g0);
                        else id[u] = ld4(a.inv_diag64, g0);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (q + u * nt >= sw.end) continue;
                const uint32_t g0 = (q + u * nt) << 2;
                Vec4<T> zv;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    zv.v[k] = T(0);
                    if (!(m[u][k] & ACTIVE)) continue;
                    xv[u].v[k] += alpha * (double)pv[u].v[k];
                    const T rn = rv[u].v[k] - al * av[u].v[k];
                    rv[u].v[k] = rn;
                    T inv = T(1);
                    if (pre) {
                        if constexpr (KIND == 0) inv = itab[m[u][k] & 63u];
                        else inv = id[u].v[k];
                    }
                    const T z = pre ? inv * rn : rn;
                    zv.v[k] = z;
                    u2[0] += (double)z * (double)rn;
                    u2[1] += (double)rn * (double)rn;
                }
                st4(x, g0, xv[u]);
                st4(r, g0, rv[u]);
                st4(zb, g0, zv);
            }
        }
    } else {
        const Sweep<ORD> sw(n, U * nt);
        for (uint32_t base = sw.start; base < sw.end; base += sw.step) {
            T pv[U], av[U], rv[U];
            double xv[U];
            unsigned m[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t gg = base + u * nt;
                const uint32_t g = gg < sw.end ? gg : base;
                if constexpr (KIND == 2) m[u] = ACTIVE;
                else m[u] = st.code[g];
                pv[u] = pc_[g];
                av[u] = apb[g];
                rv[u] = r[g];
                xv[u] = x[g];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t g = base + u * nt;
                if (g >= sw.end || !(m[u] & ACTIVE)) continue;
                x[g] = xv[u] + alpha * (double)pv[u];
                const T rn = rv[u] - al * av[u];
                r[g] = rn;
                const T z = pre ? inv_of<MIXED, KIND>(a, itab, g, m[u]) * rn : rn;
                zb[g] = z;
                u2[0] += (double)z * (double)rn;
                u2[1] += (double)rn * (double)rn;
            }
        }
    }
}

template <bool MIXED, int KIND, int NT, int U, int MINB, bool VEC, int ORD>
__global__ void __launch_bounds__(NT, MINB) k_fcg(Args a) {
    using T = typename Prec<MIXED>::T;
    mb_ctrl *c = a.ctrl;
    const bool pre = c->use_precond != 0;
    const double tol = c->tol;
    const int max_its = c->max_its;
    const double ratio = c->refine_ratio;
    T *__restrict__ r = MIXED ? (T *)a.r32 : (T *)a.r64;
    T *__restrict__ zb = MIXED ? (T *)a.z32 : (T *)a.z64;
    T *bufa = MIXED ? (T *)a.pa32 : (T *)a.pa64;
    T *bufb = MIXED ? (T *)a.pb32 : (T *)a.pb64;
    T *__restrict__ apb = MIXED ? (T *)a.ap32 : (T *)a.ap64;
    __shared__ T itab[64];
    if constexpr (KIND == 0) {
        fill_inv_table<MIXED>(a.st, itab);
        __syncthreads();
    }
    int red = 0;

    double acc[3] = {0.0, 0.0, 0.0}, s3[3];
    residual_pass<MIXED, KIND, NT, U, VEC, ORD>(a, r, bufa, pre, itab, acc);
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
        double q1[1] = {0.0}, s1[1];
        q_pass<MIXED, KIND, NT, U, VEC, ORD>(a, first, pold, pnew, zb, apb, beta, q1[0]);
        if (!grid_reduce<1, NT>(a, q1, s1, red)) return;
        const double alpha = (pre ? rz : rr) / s1[0];

        // U: x += alpha p, r -= alpha A p, z = r / diag
        double u2[2] = {0.0, 0.0}, s2[2];
        u_pass<MIXED, KIND, NT, U, VEC, ORD>(a, pcur, apb, r, zb, pre, itab, alpha, u2);
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
            if (s2[1] <= fmax(c->refine_floor, ratio * rr_ref) || its >= max_its) {
                // FP64 true residual replaces the FP32 recurrence; restart from it
                double t3[3] = {0.0, 0.0, 0.0};
                residual_pass<MIXED, KIND, NT, U, VEC, ORD>(a, r, pold, pre, itab, t3);
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

// Per-cell code bytes (kinds 0, 1) or class-table row ids (kind 2), built once
// per operator: bit q of the code says whether face q (-x,+x,-y,+y,-z,+z)
// couples the cell to an active neighbour inside the domain; bit 6 whether
// the cell itself is active.  Removed cells get code 0.
__global__ void k_codes(mb_stencil_dev st, uint8_t *code, uint16_t *rowid) {
    const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const uint32_t t = g / st.nx;
        const int i = (int)(g - t * st.nx), k = (int)(t / st.ny), j = (int)(t - (uint32_t)k * st.ny);
        if (rowid) {
            const int cx = (i == 0) ? 0 : (i == st.nx - 1 ? 2 : 1);
            const int cy = (j == 0) ? 0 : (j == st.ny - 1 ? 2 : 1);
            rowid[g] = (uint16_t)(k * 9 + cy * 3 + cx);
        }
        if (code) {
            const uint8_t *mk = st.mask;
            auto on = [&](uint32_t q) { return mk == nullptr || mk[q] != 0; };
            unsigned m = 0;
            if (on(g)) {
                m = ACTIVE;
                if (i > 0 && on(g - 1)) m |= 1u;
                if (i < st.nx - 1 && on(g + 1)) m |= 2u;
                if (j > 0 && on(g - sy)) m |= 4u;
                if (j < st.ny - 1 && on(g + sy)) m |= 8u;
                if (k > 0 && on(g - sz)) m |= 16u;
                if (k < st.nz - 1 && on(g + sz)) m |= 32u;
            }
            code[g] = (uint8_t)m;
        }
    }
}

// Jacobi inverse diagonal 1/diag per active cell, computed once per operator
// (the reference forms (1.0 / elements[0].value) at each use; the value is the
// same): alpha plus every coupled face coefficient, in the order -x, +x, -y,
// +y, -z, +z, or the centre entry of the class-table row.
__global__ void k_inv_diag(mb_stencil_dev st, double *d64, float *d32) {
    const uint32_t n = (uint32_t)st.nx * st.ny * st.nz;
    const uint32_t sy = st.nx, sz = (uint32_t)st.nx * st.ny;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        double dg64;
        float dg32;
        if (st.kind == 2) {
            const size_t row = (size_t)st.rowid[g] * 27;
            dg64 = st.table[row + 13];
            dg32 = st.table32 ? st.table32[row + 13] : (float)dg64;
        } else {
            const unsigned m = st.code[g];
            if (!(m & ACTIVE)) continue;
            double c[6];
            if (st.kind == 0) {
                c[0] = c[1] = st.cx; c[2] = c[3] = st.cy; c[4] = c[5] = st.cz;
            } else {
                c[0] = (m & 1u) ? st.fx[g - 1] : 0.0; c[1] = st.fx[g];
                c[2] = (m & 4u) ? st.fy[g - sy] : 0.0; c[3] = st.fy[g];
                c[4] = (m & 16u) ? st.fz[g - sz] : 0.0; c[5] = st.fz[g];
            }
            dg64 = st.alpha;
            float f = (float)st.alpha;
            for (int q = 0; q < 6; ++q)
                if ((m >> q) & 1u) {
                    dg64 += c[q];
                    f += (float)c[q];
                }
            dg32 = f;
        }
        if (d64) d64[g] = 1.0 / dg64;
        if (d32) d32[g] = 1.0f / dg32;
    }
}

// ---- variants -------------------------------------------------------------------

struct Variant {
    const void *fn;
    int threads;   // at most this many per block
    int groups;    // 1 = four cells per thread
    int cells;     // units (cells or groups) each thread takes per round
};

// (threads per block, cells per thread per round, resident blocks per SM,
// four-cell groups); the group variants need nx to be a multiple of 4
#define MB_SHAPES(K, O)                                                                                          \
    {(const void *)k_fcg<MIXED, K, 1024, 1, 1, false, O>, 1024, 0, 1},                                      \
        {(const void *)k_fcg<MIXED, K, 1024, 1, 2, false, O>, 1024, 0, 1},                                  \
        {(const void *)k_fcg<MIXED, K, 512, 2, 2, false, O>, 512, 0, 2},                                    \
        {(const void *)k_fcg<MIXED, K, 512, 1, 4, false, O>, 512, 0, 1},                                    \
        {(const void *)k_fcg<MIXED, K, 256, 2, 4, false, O>, 256, 0, 2},                                    \
        {(const void *)k_fcg<MIXED, K, 1024, 1, 1, true, O>, 1024, 1, 1},                                   \
        {(const void *)k_fcg<MIXED, K, 512, 1, 2, true, O>, 512, 1, 1},                                     \
        {(const void *)k_fcg<MIXED, K, 256, 1, 4, true, O>, 256, 1, 1},                                     \
        {(const void *)k_fcg<MIXED, K, 512, 2, 1, true, O>, 512, 1, 2},                                     \
        {(const void *)k_fcg<MIXED, K, 256, 2, 2, true, O>, 256, 1, 2},                                     \
        {(const void *)k_fcg<MIXED, K, 512, 1, 1, true, O>, 512, 1, 1},                                     \
        {(const void *)k_fcg<MIXED, K, 256, 1, 2, true, O>, 256, 1, 1}
// variants 0..11: each block sweeps its own range; 12..23: the same shapes
// with the interleaved sweep.  The last two shapes give a thread 128
// registers, enough for every row load of a 27-point group in flight.
#define MB_VARIANTS(K) MB_SHAPES(K, 0), MB_SHAPES(K, 1)

constexpr int NUM_VARIANTS = 24;

template <bool MIXED>
static Variant variant_of(int kind, int v) {
    static const Variant t0[NUM_VARIANTS] = {MB_VARIANTS(0)};
    static const Variant t1[NUM_VARIANTS] = {MB_VARIANTS(1)};
    static const Variant t2[NUM_VARIANTS] = {MB_VARIANTS(2)};
    return kind == 0 ? t0[v] : (kind == 1 ? t1[v] : t2[v]);
}
#undef MB_VARIANTS
#undef MB_SHAPES

static Variant variant(int mixed, int kind, int v) {
    return mixed ? variant_of<true>(kind, v) : variant_of<false>(kind, v);
}

}  // namespace fcg
}  // namespace mb

using namespace mb::fcg;

extern "C" int mbk_fcg_variants(int kind) {
    (void)kind;
    return NUM_VARIANTS;
}

// Whether variant v runs four-cell groups (usable only when nx % 4 == 0).
extern "C" int mbk_fcg_variant_groups(int v) {
    return v >= 0 && v < NUM_VARIANTS ? variant(0, 0, v).groups : 0;
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

extern "C" int mbk_stencil_codes(const mb_stencil_dev *st, uint8_t *code, uint16_t *rowid, cudaStream_t s) {
    k_codes<<<592, 256, 0, s>>>(*st, code, rowid);
    return (int)cudaGetLastError();
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
    a.ap64 = p->ap64; a.ap32 = p->ap32;
    a.inv_diag64 = p->inv_diag64; a.inv_diag32 = p->inv_diag32;
    a.partials = p->partials; a.ctrl = p->ctrl; a.bar = p->bar; a.status = p->status;
    const Variant var = variant(p->mixed, p->st.kind, p->variant);
    // the arrival counter starts from zero in every launch
    cudaError_t e = cudaMemsetAsync(p->bar, 0, 2 * sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    // Block size: the fewest threads (a multiple of 32, at most the variant's)
    // that cover each block's range in the same whole number of rounds as the
    // variant's full block, so that no round runs partly empty.
    const unsigned long long n = (unsigned long long)p->st.nx * p->st.ny * p->st.nz;
    const unsigned long long units = var.groups ? n / 4 : n;
    const unsigned long long chunk = ((units + p->blocks - 1) / p->blocks + 31) & ~31ULL;
    const unsigned long long per_round = (unsigned long long)var.threads * var.cells;
    const unsigned long long rounds = chunk ? (chunk + per_round - 1) / per_round : 1;
    unsigned long long threads = ((chunk + rounds * var.cells - 1) / (rounds * var.cells) + 31) & ~31ULL;
    if (threads < 32) threads = 32;
    if (threads > (unsigned long long)var.threads) threads = var.threads;
    void *args[] = {&a};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p->blocks);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelExC(&cfg, var.fn, args);
}

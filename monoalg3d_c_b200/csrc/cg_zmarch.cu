// Persistent Jacobi-PCG for the 27-point operator of fibres rotating through
// the thickness (kind 2: rows from the per-plane class table), marching
// through z with every plane of the stencil's input staged in shared memory
// by the Tensor Memory Accelerator.  Same Krylov recurrences, refinement rule
// and stopping test as the flat kernel (cg_flat.cu), which follow
// cpu_conjugate_gradient (src/linear_system_solver_library/linear_system_solver.c:47-183).
//
// Why: on the flat kernel each thread gathers the nine rows of a 27-point
// stencil from L1/L2 with a dependent row -> coefficient -> FMA chain, and the
// Q pass runs at a quarter of the DRAM rate its bytes allow.  Here a block
// owns a tile of 128 x W cells (a warp per x-row, four cells per lane) over a
// range of planes and walks it plane by plane:
//
//   TMA   cp.async.bulk.tensor.3d loads the next planes' tiles (with a halo
//         of 4 cells in x -- the 16-byte alignment of the box -- and 1 in y;
//         cells outside the grid read as zeros) into S stage buffers, each
//         completed on its own mbarrier, up to S planes ahead of the compute;
//   form  each staged plane is turned into the stencil's input in a ring of
//         four planes: the direction p = r / diag + beta p_old (Q pass; the
//         Jacobi z is never stored) or x itself (residual pass); the Q pass
//         stores the new direction's tile cells to global memory here;
//   apply the output plane k reads planes k-1, k, k+1 of the ring: nine rows
//         of four cells per lane (one 16-byte shared load each, the values
//         left and right of the lane's four cells by warp shuffle), summed
//         in the table's entry order (the same sums as the flat kernel).
//
// Each stage buffer and each ring plane is rewritten only after the block
// barrier that follows its last use, so one __syncthreads per plane orders
// the pipeline.  A block walks either an equal share of the (tile, plane)
// pairs (balanced ranges) or units (x tile, y tile, z chunk) taken in turn;
// either way the blocks work on neighbouring tiles at nearby planes and the
// halo rows they share are mostly read from L2.
//
// Per iteration, ring and window forms: Q (stencil pass: reads r, p_old;
// writes p, A p; p.Ap), then U (streaming pass: x += alpha p, r -= alpha A p,
// r.z and r.r with z = r / diag formed and dropped).  Fused form (mixed):
// one stencil pass that updates r from the staged r and A p, forms p, applies
// the previous x update and sums seven products for one reduction (see
// fpass).  The FP64 residual b - A x (start and refinements) is a stencil
// pass over x.  Jacobi 1/diag comes from a per-plane
// table of the nine row classes (1 / the class row's diagonal entry, the value
// the flat kernel stores per cell).
//
// The tensor maps live in global memory (64-byte aligned, written from the
// host before any launch that reads them).  Every wait is bounded: an
// mbarrier wait that has not completed after SPIN_LIMIT polls makes the block
// record MB_ERR_CUDA in the status word, wait (again bounded) for its copies
// still in flight and leave the kernel; the other blocks then time out at
// their next grid reduction and leave too.
#include <cuda.h>
#include <cstdlib>
#include <cstring>
#include "cg_common.cuh"

namespace mb {
namespace zcg {

using fcg::Args;
using fcg::grid_reduce;
using fcg::SPIN_LIMIT;

constexpr int TX = 128;            // tile width in x: 32 lanes x 4 cells
constexpr int HX = 4;              // x halo per side (16 bytes of FP32)
constexpr int WX = TX + 2 * HX;    // staged row length
constexpr int RING = 4;            // ring planes
constexpr int MAPS = 8;            // tensor maps per variant

// Division by a fixed divisor d as a multiply and shifts (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994,
// round-up form): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> 1)) >> (l - 1) for t = mulhi(m, n), every 32-bit n.
struct FastDiv {
    uint32_t d, m, l;
    __device__ __forceinline__ uint32_t div(uint32_t n) const {
        if (d == 1) return n;
        const uint32_t t = __umulhi(m, n);
        return (t + ((n - t) >> 1)) >> (l - 1);
    }
};

struct ZArgs {
    const double *inv64;           // [nz][9] Jacobi 1/diag per plane and class
    const float *inv32;
    // [nz][PTAB] FP32: a plane's nine class rows (padded to CROW entries),
    // its nine Jacobi values at JOFF, zero padding -- one 16-byte-aligned
    // block per plane for the bulk copy of the window Q pass
    const float *ptab32;
    // tensor maps of r, p (buffer a), p (buffer b) and x, in global memory
    const CUtensorMap *maps;
    int tiles_x, tiles_y, chunks;
    // 1: each block walks its own share of the (tile, plane) pairs in
    // tile-major order (balanced ranges, below); 0: blocks take units of
    // whole z chunks in turn (the window Q pass's form)
    int balanced;
    FastDiv by_gx, by_ny;          // n / (nx / 4), n / ny
};

__host__ __device__ constexpr int r128(int b) { return (b + 127) / 128 * 128; }

constexpr int TSLOTS = 4;          // per-plane table slots
constexpr int TROW = 9 * 27 + 9;   // one plane in global memory: 9 class rows of 27 entries, 9 Jacobi values
// In shared memory each class row is padded to CROW entries, so that a row
// starts on a 16-byte boundary and its coefficients load as vectors (one
// broadcast wavefront per four FP32 / two FP64 entries); the Jacobi values
// follow at JOFF.
constexpr int CROW = 28;
constexpr int JOFF = 9 * CROW;
constexpr int TSLOT = JOFF + 12;   // entries per plane slot (a multiple of 4)
constexpr int PTAB = TSLOT;        // the same block in global memory (FP32, 16-byte multiple)
constexpr int QDLY = 2;            // window Q pass: the stage of entry e is refilled at step e + QDLY

// Iteration forms (the kernel's MODE): the ring Q pass and the U pass; the
// window Q pass and the U pass; the fused pass (mixed only: one stencil pass
// and one reduction per iteration).
enum { QRING = 0, QWIN = 1, FUSED = 2 };

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <typename T, int W, int S, int MODE = QRING>
struct Lay {
    static constexpr int H = W + 2;                         // staged rows
    static constexpr int ELEMS = H * WX;                    // one staged plane
    static constexpr int ARR = r128(ELEMS * (int)sizeof(T));
    static constexpr int XARR = r128(ELEMS * 8);            // a staged plane of doubles (x)
    // window Q pass: r, p_old and the plane's table (FP32) per stage
    static constexpr int QSTAGE = (MODE == QWIN && sizeof(T) == 4) ? 2 * ARR + r128(PTAB * 4) : 0;
    // fused pass: r, A p and p_old; its residual pass: x and p
    static constexpr int FSTAGE = MODE == FUSED ? cmax(3 * ARR, XARR + ARR) : 0;
    static constexpr int STAGE = cmax(cmax(2 * ARR, XARR), cmax(QSTAGE, FSTAGE));
    // ring planes hold doubles (residual pass); in the fused pass a ring
    // plane holds the direction p and then the residual r
    static constexpr int RPLANE = MODE == FUSED ? cmax(XARR, 2 * ARR) : XARR;
    static constexpr int BARS = 128;
    // the coefficient rows and Jacobi values of up to four planes, both
    // precisions (the residual pass applies the FP64 rows)
    static constexpr int TABS = r128(TSLOTS * TSLOT * 8) + r128(TSLOTS * TSLOT * 4);
    // + 128: the dynamic shared memory base is aligned up to 128 bytes at run
    // time (bulk tensor copies write to 128-byte-aligned shared addresses)
    static constexpr int BYTES = BARS + TABS + S * STAGE + RING * RPLANE + 128;
};

// ---- PTX: mbarrier and bulk tensor copies ---------------------------------------

__device__ __forceinline__ uint32_t s32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// The shared-window address of p, computed where the compiler cannot apply
// what it assumes about p's alignment.
__device__ __forceinline__ uint32_t smem_addr_opaque(const void *p) {
    uint32_t a;
    asm volatile("{\n\t.reg .u64 t;\n\tcvta.to.shared.u64 t, %1;\n\tcvt.u32.u64 %0, t;\n\t}" : "=r"(a) : "l"(p));
    return a;
}

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(s32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity) {
    long long spins = 0;
    while (!mbar_try_wait(b, parity)) {
        if (++spins > SPIN_LIMIT) return false;
        if (spins > 64) __nanosleep(32);
    }
    return true;
}
// Orders this thread's earlier generic-proxy accesses (and those it has
// acquired from other threads) before its later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s32(b)) : "memory");
}
// 1-D bulk copy global -> shared (16-byte aligned ends, size a multiple of 16)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     s32(dst)),
                 "l"(src), "r"(bytes), "r"(s32(bar))
                 : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(s32(dst)),
        "l"(map), "r"(s32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// ---- vectors of four cells ---------------------------------------------------------

template <typename T>
struct V4 { T v[4]; };

__device__ __forceinline__ V4<float> ld4(const float *p) {
    const float4 f = *reinterpret_cast<const float4 *>(p);
    return {{f.x, f.y, f.z, f.w}};
}
__device__ __forceinline__ V4<double> ld4(const double *p) {
    const double2 a = *reinterpret_cast<const double2 *>(p);
    const double2 b = *reinterpret_cast<const double2 *>(p + 2);
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float *p, const V4<float> &v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v.v[0], v.v[1], v.v[2], v.v[3]);
}
__device__ __forceinline__ void st4(double *p, const V4<double> &v) {
    *reinterpret_cast<double2 *>(p) = make_double2(v.v[0], v.v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v.v[2], v.v[3]);
}
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <bool MIXED>
struct Prec { using T = double; };
template <>
struct Prec<true> { using T = float; };

// row class of a cell along one axis: 0 on the low face, 2 on the high face
__device__ __forceinline__ int axis_class(int i, int n) { return i <= 0 ? 0 : (i >= n - 1 ? 2 : 1); }

template <typename T>
__device__ __forceinline__ const T *inv_table(const ZArgs &z);
template <>
__device__ __forceinline__ const float *inv_table<float>(const ZArgs &z) { return z.inv32; }
template <>
__device__ __forceinline__ const double *inv_table<double>(const ZArgs &z) { return z.inv64; }

template <typename T>
__device__ __forceinline__ T coef(const mb_stencil_dev &st, size_t idx) {
    if constexpr (sizeof(T) == 8) return __ldg(st.table + idx);
    else return __ldg(st.table32 + idx);
}

// ---- units ----------------------------------------------------------------------

struct Unit {
    int x0, y0, k0, k1;
};

// Tile t (x fastest) over planes k0..k1-1.
template <int W>
__device__ __forceinline__ Unit tile_unit(const ZArgs &z, int t, int k0, int k1) {
    const int ty = t / z.tiles_x;
    return Unit{(t - ty * z.tiles_x) * TX, ty * W, k0, k1};
}

template <int W>
__device__ __forceinline__ Unit unit_of(const ZArgs &z, int nz, int u) {
    const int tx = u % z.tiles_x;
    const int t = u / z.tiles_x;
    const int ty = t % z.tiles_y;
    const int c = t / z.tiles_y;
    Unit U;
    U.x0 = tx * TX;
    U.y0 = ty * W;
    U.k0 = (int)(((long long)c * nz) / z.chunks);
    U.k1 = (int)(((long long)(c + 1) * nz) / z.chunks);
    return U;
}

// Pipeline state carried across units and passes: the parity each stage's
// mbarrier completes next.
struct Pipe {
    uint32_t phase;
};

// A class row (CROW entries, 16-byte aligned, in shared memory) into registers
// by vector loads.
__device__ __forceinline__ void load_row(const float *row, float (&cc)[CROW]) {
#pragma unroll
    for (int q = 0; q < CROW; q += 4) {
        const float4 v = *reinterpret_cast<const float4 *>(row + q);
        cc[q] = v.x;
        cc[q + 1] = v.y;
        cc[q + 2] = v.z;
        cc[q + 3] = v.w;
    }
}
__device__ __forceinline__ void load_row(const double *row, double (&cc)[CROW]) {
#pragma unroll
    for (int q = 0; q < CROW; q += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(row + q);
        cc[q] = v.x;
        cc[q + 1] = v.y;
    }
}

// The 27-point product for the lane's four cells of row j, from ring planes
// lo (k-1), mid (k), hi (k+1) (row stride WX, staged row h = the tile row +
// 1) and the plane's class rows ct (9 rows of 27 entries in shared memory).
// Every cell is first summed with the row of its y class and the interior x
// class (the same row for the whole warp); a cell on an x face (i = 0 or
// nx - 1) is also summed with its own row, which replaces its first sum.
// Sums run in entry order.  DENSE: every one of the 27 entries is applied -- the table holds
// zeros where the operator has none, and fma(0, v, s) = s, so the sums are
// those of the sparse form -- as straight-line code whose shared loads the
// compiler can issue ahead of the arithmetic (measured faster than skipping
// the entries that are zero in every row, st.nzmask, in both precisions).
// All 32 lanes call it together.
// FACE: some lane of the warp holds a cell on an x face (warp-uniform); its
// own row's sum runs beside the others in the same entry order, from the
// same values (the face cell's neighbours are already in the lane's
// registers), instead of a pass over shared memory after them.
template <typename R, int W, bool DENSE, bool FACE>
__device__ __forceinline__ V4<R> apply27_rows(const mb_stencil_dev &st, const R *lo, const R *mid, const R *hi,
                                              const R *ct, int e, int cy, int w, int lane) {
    const R *cm = ct + (cy * 3 + 1) * CROW;
    // the face row of a lane holding a face cell (lanes without one read
    // the low face's row and drop the sum)
    const R *ce = ct + (cy * 3 + (e == 3 ? 2 : 0)) * CROW;
    const uint32_t mask = DENSE ? 0x7ffffffu : st.nzmask;
    // FP32: the row in registers, loaded as vectors; FP64 reads each entry
    // where it is used (its 28 values would take 56 registers)
    R cc[sizeof(R) == 4 ? CROW : 1];
    if constexpr (sizeof(R) == 4) load_row(cm, cc);
    R acc[4] = {R(0), R(0), R(0), R(0)};
    R af = R(0);
    const int off = HX + 4 * lane;
    // the value beyond the tile's row: left of it for lane 0, right of it
    // for the others (used by lane 31) -- two distinct addresses in
    // different banks, one shared-memory wavefront per row (each lane
    // reading its own neighbour would take four to eight)
    const int hoff = lane == 0 ? HX - 1 : HX + TX;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz) {
        const R *pl = dz < 0 ? lo : (dz == 0 ? mid : hi);
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            const unsigned rb = (mask >> ((dz + 1) * 9 + (dy + 1) * 3)) & 7u;
            if (!rb) continue;
            const R *rowb = pl + (w + 1 + dy) * WX;
            const R *rowp = rowb + off;
            const V4<R> m4 = ld4(rowp);
            const R he = rowb[hoff];
            const R sl = __shfl_up_sync(0xffffffffu, m4.v[3], 1);
            const R sr = __shfl_down_sync(0xffffffffu, m4.v[0], 1);
            R wv[6];
            // (selects, not a branch: a branch per row keeps the compiler
            // from scheduling the rows' loads ahead, measured slower)
            wv[0] = lane == 0 ? he : sl;
            wv[5] = lane == 31 ? he : sr;
#pragma unroll
            for (int c = 0; c < 4; ++c) wv[c + 1] = m4.v[c];
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (!((rb >> (dx + 1)) & 1u)) continue;
                const int q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                R cq;
                if constexpr (sizeof(R) == 4) cq = cc[q];
                else cq = cm[q];
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[c] = fma(cq, wv[c + 1 + dx], acc[c]);
                // the face cell (e = 0 or 3) and its neighbours e + dx
                if constexpr (FACE) af = fma(ce[q], e == 3 ? wv[4 + dx] : wv[1 + dx], af);
            }
        }
    }
    if constexpr (FACE) {
        if (e == 0) acc[0] = af;
        else if (e == 3) acc[3] = af;
    }
    V4<R> out;
#pragma unroll
    for (int c = 0; c < 4; ++c) out.v[c] = acc[c];
    return out;
}

template <typename R, int W, bool DENSE = true>
__device__ __forceinline__ V4<R> apply27(const mb_stencil_dev &st, const R *lo, const R *mid, const R *hi,
                                         const R *ct, int i0, int j, int w, int lane) {
    const int cy = axis_class(j, st.ny);
    // the lane's cell on an x face, if any: the first of its four on the
    // low face, the last on the high face
    const int e = i0 == 0 ? 0 : (i0 + 3 == st.nx - 1 ? 3 : -1);
    if (__any_sync(0xffffffffu, e >= 0)) return apply27_rows<R, W, DENSE, true>(st, lo, mid, hi, ct, e, cy, w, lane);
    return apply27_rows<R, W, DENSE, false>(st, lo, mid, hi, ct, e, cy, w, lane);
}

// The 27-point product for the lane's four cells of row j of plane k from a
// register window: win[pz][ry] = the lane's four values of plane k - 1 + pz,
// row j - 1 + ry; hx[pz][ry] = the value beyond the tile's edge (left of the
// tile in lane 0, right of it in lane 31); tb = plane k's nine class rows.
// The same sums as apply27: entry order, the warp's interior row for every
// cell, then the cells on an x face of the grid with their own rows (their
// neighbours outside the grid are zero, as the staged halo is there).
template <typename R>
__device__ __forceinline__ V4<R> apply_w(const mb_stencil_dev &st, const V4<R> (&win)[3][3], const R (&hx)[3][3],
                                         const float *tb, int i0, int j, int lane) {
    const int cy = axis_class(j, st.ny);
    float cc[CROW];
    load_row(tb + (cy * 3 + 1) * CROW, cc);
    const uint32_t mask = 0x7ffffffu;      // dense, as apply27 in FP32
    R acc[4] = {R(0), R(0), R(0), R(0)};
#pragma unroll
    for (int pz = 0; pz < 3; ++pz) {
#pragma unroll
        for (int ry = 0; ry < 3; ++ry) {
            const unsigned rb = (mask >> (pz * 9 + ry * 3)) & 7u;
            if (!rb) continue;
            const V4<R> &m4 = win[pz][ry];
            const R sl = __shfl_up_sync(0xffffffffu, m4.v[3], 1);
            const R sr = __shfl_down_sync(0xffffffffu, m4.v[0], 1);
            R wv[6];
            wv[0] = lane == 0 ? hx[pz][ry] : sl;
            wv[5] = lane == 31 ? hx[pz][ry] : sr;
#pragma unroll
            for (int c = 0; c < 4; ++c) wv[c + 1] = m4.v[c];
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                if (!((rb >> (dx + 1)) & 1u)) continue;
                const R c0 = (R)cc[pz * 9 + ry * 3 + (dx + 1)];
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[c] = fma(c0, wv[c + 1 + dx], acc[c]);
            }
        }
    }
    // cells on an x face: only the lanes holding one take this branch
    const int e = i0 == 0 ? 0 : (i0 + 3 == st.nx - 1 ? 3 : -1);
    if (e >= 0) {
        const float *ce = tb + (cy * 3 + axis_class(i0 + e, st.nx)) * CROW;
        R a = R(0);
#pragma unroll
        for (int pz = 0; pz < 3; ++pz) {
#pragma unroll
            for (int ry = 0; ry < 3; ++ry) {
                const V4<R> &m4 = win[pz][ry];
                // the face cell's neighbours dx = -1, 0, +1 (zero outside the grid)
                const R lo[3] = {R(0), m4.v[0], m4.v[1]};
                const R hi[3] = {m4.v[2], m4.v[3], R(0)};
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    const int q = pz * 9 + ry * 3 + dx;
                    a = fma((R)ce[q], e == 0 ? lo[dx] : hi[dx], a);
                }
            }
        }
        if (e == 0) acc[0] = a;
        else acc[3] = a;
    }
    V4<R> out;
#pragma unroll
    for (int c = 0; c < 4; ++c) out.v[c] = acc[c];
    return out;
}

// One stencil pass over every unit of this block.  issue(U, m, stage, bar)
// (thread 0) starts the copies of plane m of unit U into a stage buffer;
// form(U, m, stage, ring) turns a staged plane into ring plane input;
// out(U, k, lo, mid, hi) produces output plane k.  Returns false after a wait
// timed out (the status word is set).
//
// Plane v of a unit (plane k0 - 1 + v) has its coefficient rows and Jacobi
// values in table slot v % 4: read from global memory into registers
// (tabs.fetch) in step v - 2, stored to the slot (tabs.put) in step v - 1
// before that step's barrier (the prologue does both for v = 0 and fetches
// v = 1), read by the form of step v and the output of step v + 1, and
// rewritten in step v + 3 -- after the barrier of step v + 2, which every
// reader of step v + 1 has passed.  The fetch one step ahead keeps the
// global load's latency off the path to the barrier.
template <int W, int S, typename IssueF, typename TabF, typename FormF, typename OutF>
__device__ __forceinline__ bool zpass(const ZArgs &z, const Args &a, unsigned char *smem, int tabs_bytes,
                                      int stage_bytes, int rplane_bytes, Pipe &pp, IssueF issue, TabF &tabs,
                                      FormF form, OutF out) {
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    unsigned char *stage0 = smem + 128 + tabs_bytes;
    unsigned char *ring0 = stage0 + (size_t)S * stage_bytes;
    const int nz = a.st.nz;
    auto run = [&](const Unit &U) -> bool {
        const int P = U.k1 - U.k0 + 2;     // planes k0-1 .. k1
        if (threadIdx.x == 0) {
            fence_proxy_async();
            for (int u = 0; u < S && u < P; ++u) issue(U, U.k0 - 1 + u, stage0 + (size_t)u * stage_bytes, &bars[u]);
        }
        tabs.fetch(U.k0 - 1);
        tabs.put(0);
        if (P > 1) tabs.fetch(U.k0);
        __syncthreads();
        for (int u = 0; u < P; ++u) {
            const int s = u % S;
            const unsigned par = (pp.phase >> s) & 1u;
            const bool ok = mbar_wait(&bars[s], par);
            pp.phase ^= 1u << s;
            if (u + 1 < P) tabs.put((u + 1) % TSLOTS);
            if (u + 2 < P) tabs.fetch(U.k0 + u + 1);
            form(U, U.k0 - 1 + u, u % TSLOTS, stage0 + (size_t)s * stage_bytes,
                 ring0 + (size_t)(u & (RING - 1)) * rplane_bytes);
            if (!__syncthreads_and(ok)) {
                // copies this block started and has not waited for: plane u
                // (whose wait gave up) and the ones issued after it
                if (threadIdx.x == 0) {
                    atomicExch(a.status, MB_ERR_CUDA);
                    for (int v = u; v < P && v < u + S; ++v) {
                        const int sv = v % S;
                        const unsigned pv = v == u ? par : ((pp.phase >> sv) & 1u);
                        (void)mbar_wait(&bars[sv], pv);
                    }
                }
                __syncthreads();
                return false;
            }
            if (threadIdx.x == 0 && u + S < P) issue(U, U.k0 - 1 + u + S, stage0 + (size_t)s * stage_bytes, &bars[s]);
            if (u >= 2) {
                out(U, U.k0 + u - 2, (u - 1) % TSLOTS, ring0 + (size_t)((u - 2) & (RING - 1)) * rplane_bytes,
                    ring0 + (size_t)((u - 1) & (RING - 1)) * rplane_bytes,
                    ring0 + (size_t)(u & (RING - 1)) * rplane_bytes);
            }
        }
        __syncthreads();
        return true;
    };
    if (z.balanced) {
        // Block b walks the pairs [b N / G, (b + 1) N / G) of the N = tiles x nz
        // (tile, plane) pairs in tile-major order, so every block has the same
        // number of planes (within one) plus two halo planes per tile it
        // touches.  Its tiles are walked last first: the block that ends a
        // tile's range starts at plane 0 of the next tile, so every tile's
        // plane k is reached within nz - N / G steps of step k and the halo
        // rows neighbouring tiles share are still read from L2.
        const long long N = (long long)z.tiles_x * z.tiles_y * nz;
        const long long s0 = (long long)blockIdx.x * N / gridDim.x;
        const long long s1 = (long long)(blockIdx.x + 1) * N / gridDim.x;
        if (s1 > s0) {
            const int tf = (int)(s0 / nz), tl = (int)((s1 - 1) / nz);
            for (int t = tl; t >= tf; --t) {
                const long long base = (long long)t * nz;
                const int k0 = s0 > base ? (int)(s0 - base) : 0;
                const int k1 = s1 < base + nz ? (int)(s1 - base) : nz;
                if (!run(tile_unit<W>(z, t, k0, k1))) return false;
            }
        }
        return true;
    }
    const int units = z.tiles_x * z.tiles_y * z.chunks;
    for (int un = blockIdx.x; un < units; un += gridDim.x)
        if (!run(unit_of<W>(z, nz, un))) return false;
    return true;
}

// A plane's class rows and Jacobi values (TROW entries per precision), each
// thread holding the entries e = threadIdx.x + NT i between fetch and put.
template <int NT>
struct Tabs {
    static constexpr int PER = (TROW + NT - 1) / NT;
    double *tab64;
    float *tab32;
    const double *table;
    const float *table32;
    const double *inv64;
    const float *inv32;
    int nz;
    double h64[PER];
    float h32[PER];
    __device__ __forceinline__ void fetch(int m) {
        const int mm = m < 0 ? 0 : (m >= nz ? nz - 1 : m);
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int e = threadIdx.x + NT * i;
            if (e < TROW) {
                const size_t src = e < 243 ? (size_t)mm * 243 + e : (size_t)mm * 9 + (e - 243);
                h64[i] = e < 243 ? __ldg(table + src) : __ldg(inv64 + src);
                h32[i] = e < 243 ? __ldg(table32 + src) : __ldg(inv32 + src);
            }
        }
    }
    __device__ __forceinline__ void put(int slot) {
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int e = threadIdx.x + NT * i;
            if (e < TROW) {
                const int row = e / 27;
                const int d = e < 243 ? row * CROW + (e - row * 27) : JOFF + (e - 243);
                tab64[slot * TSLOT + d] = h64[i];
                tab32[slot * TSLOT + d] = h32[i];
            }
        }
    }
};

// ---- the solve ----------------------------------------------------------------

template <bool MIXED, int W, int S, int MINB, int MODE>
__global__ void __launch_bounds__(32 * W, MINB) k_zcg(Args a, ZArgs z) {
    using T = typename Prec<MIXED>::T;
    using L = Lay<T, W, S, MODE>;
    static_assert(MODE != FUSED || MIXED, "the fused pass is the mixed form's");
    static_assert(S <= 4, "the barrier area holds 4 + 4 + 4 mbarriers");
    // Dynamic shared memory starts after the static reduction arrays of
    // grid_reduce, at an offset aligned to 16 bytes only; it is declared
    // with that alignment (a larger declared one would let the compiler
    // fold the adjustment below away) and aligned up to 128 bytes here, the
    // address taken through an asm the compiler cannot see through.
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t raw = smem_addr_opaque(smem_raw);
    unsigned char *smem = smem_raw + ((128u - (raw & 127u)) & 127u);
    const mb_stencil_dev &st = a.st;
    mb_ctrl *c = a.ctrl;
    const bool pre = c->use_precond != 0;
    const double tol = c->tol;
    const int max_its = c->max_its;
    const double ratio = c->refine_ratio;
    T *__restrict__ r = MIXED ? (T *)a.r32 : (T *)a.r64;
    T *bufa = MIXED ? (T *)a.pa32 : (T *)a.pa64;
    T *bufb = MIXED ? (T *)a.pb32 : (T *)a.pb64;
    T *__restrict__ apb = MIXED ? (T *)a.ap32 : (T *)a.ap64;
    const T *invt = inv_table<T>(z);
    const int nx = st.nx, ny = st.ny, nz = st.nz;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;

    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    // never issue a copy to a misaligned buffer or through a misaligned map
    if ((smem_addr_opaque(smem) & 127u) || (reinterpret_cast<uintptr_t>(z.maps) & 63u)) {
        if (threadIdx.x == 0) atomicExch(a.status, MB_ERR_CUDA);
        return;
    }
    const CUtensorMap *tm_r = z.maps, *tm_pa = z.maps + 1, *tm_pb = z.maps + 2, *tm_x = z.maps + 3;
    if (threadIdx.x == 0) {
        // the maps were written by a copy from the host: acquire them for the
        // tensor-map proxy before the first bulk copy reads them
        for (int q = 0; q < (MODE == FUSED ? MAPS : 4); ++q)
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(z.maps + q) : "memory");
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        // window Q pass: full (the copies of a stage) and empty (every warp
        // done with it) barriers
        for (int s = 0; s < S; ++s) {
            mbar_init(&bars[4 + s], 1);
            mbar_init(&bars[8 + s], W);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    Pipe pp{0u};
    int red = 0;

    // per-plane tables in shared memory (see zpass): slot s holds a plane's
    // nine class rows (27 entries each) and then its nine Jacobi values, in
    // FP64 (tab64) and FP32 (tab32)
    double *tab64 = reinterpret_cast<double *>(smem + 128);
    float *tab32 = reinterpret_cast<float *>(smem + 128 + r128(TSLOTS * TSLOT * 8));
    Tabs<32 * W> tabs{tab64, tab32, st.table, st.table32, z.inv64, z.inv32, nz};
    auto tabT = [&](int slot) -> const T * {
        if constexpr (sizeof(T) == 8) return tab64 + slot * TSLOT;
        else return tab32 + slot * TSLOT;
    };

    // ---- residual pass: r = b - A x (FP64), partials r.z, r.r, r64.r64 ----------
    // With pk (the fused form's refinement) the stencil's input is x + alx pk,
    // the update of x the fused form has not yet applied, formed from the
    // staged x and pk in the same FP64 fma that later applies it to x.  The
    // FP32 residual goes to rdst.
    auto residual = [&](T *rdst, const T *pk, double alx, double (&acc)[3]) -> bool {
        const CUtensorMap *mpk = pk == bufa ? tm_pa : tm_pb;
        auto issue = [&](const Unit &U, int m, unsigned char *stg, uint64_t *bar) {
            mbar_expect_tx(bar, (unsigned)(L::ELEMS * 8) + (pk ? (unsigned)(L::ELEMS * sizeof(T)) : 0u));
            tma_load_3d(stg, tm_x, bar, U.x0 - HX, U.y0 - 1, m);
            if (pk) tma_load_3d(stg + L::XARR, mpk, bar, U.x0 - HX, U.y0 - 1, m);
        };
        auto form = [&](const Unit &, int, int, unsigned char *stg, unsigned char *rp) {
            const double2 *src = reinterpret_cast<const double2 *>(stg);
            double2 *dst = reinterpret_cast<double2 *>(rp);
            if (!pk) {
                for (int e = threadIdx.x; e < L::ELEMS / 2; e += blockDim.x) dst[e] = src[e];
            } else {
                const T *ps = reinterpret_cast<const T *>(stg + L::XARR);
                for (int e = threadIdx.x; e < L::ELEMS / 2; e += blockDim.x) {
                    const double2 xv = src[e];
                    dst[e] = make_double2(fma(alx, (double)ps[2 * e], xv.x), fma(alx, (double)ps[2 * e + 1], xv.y));
                }
            }
        };
        auto out = [&](const Unit &U, int k, int ts, unsigned char *lo, unsigned char *mid, unsigned char *hi) {
            const int j = U.y0 + w, i0 = U.x0 + 4 * lane;
            if (j >= ny) return;                     // warp-uniform
            const size_t g0 = (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * k);
            // the right-hand side's cells, loaded before the product so that
            // the global load's latency runs under it
            V4<double> bv = {{0.0, 0.0, 0.0, 0.0}};
            if (i0 < nx) bv = ld4(a.b ? a.b + g0 : a.vstar + g0);
            const double *ct = tab64 + ts * TSLOT;
            const V4<double> ax = apply27<double, W>(st, reinterpret_cast<const double *>(lo),
                                                     reinterpret_cast<const double *>(mid),
                                                     reinterpret_cast<const double *>(hi), ct, i0, j, w, lane);
            if (i0 >= nx) return;
            const T *iv = tabT(ts) + JOFF + axis_class(j, ny) * 3;
            V4<T> rv;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double bb = a.b ? bv.v[e] : st.alpha * bv.v[e];
                const double r64 = bb - ax.v[e];
                const T rt = (T)r64;
                const T zz = pre ? mul_rn(iv[axis_class(i0 + e, nx)], rt) : rt;
                rv.v[e] = rt;
                acc[0] += (double)rt * (double)zz;
                acc[1] += (double)rt * (double)rt;
                acc[2] += r64 * r64;
            }
            st4(rdst + g0, rv);
            // the fused solve keeps A x of its refinements: the last one is A x
            // of the solution, the next solve's starting product
            if (pk && a.w) st4(a.w + g0, ax);
        };
        return zpass<W, S>(z, a, smem, L::TABS, L::STAGE, L::RPLANE, pp, issue, tabs, form, out);
    };

    // ---- initial residual from the stored product (fused, mixed): r = b - w ----
    // w = A x as the previous solve's last residual pass formed it for the x
    // this solve starts from (the same FP64 sums), so r is the residual the
    // stencil pass would give, for 20 streamed bytes per cell instead of a
    // stencil pass.  Partials r.z, r.r, r64.r64 as there.
    auto residual_w = [&](T *rdst, double (&acc)[3]) {
        const unsigned gx = (unsigned)nx >> 2;
        const unsigned groups = gx * (unsigned)ny * (unsigned)nz;
        for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
            const size_t g0 = (size_t)q << 2;
            const V4<double> bv = ld4(a.b ? a.b + g0 : a.vstar + g0);
            const V4<double> wv = ld4(a.w + g0);
            const unsigned t = z.by_gx.div(q);
            const int i0 = (int)(q - t * gx) << 2;
            const unsigned kk = z.by_ny.div(t);
            const int k = (int)kk, j = (int)(t - kk * (unsigned)ny);
            const T *irow = invt + k * 9 + axis_class(j, ny) * 3;
            V4<T> rv;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double bb = a.b ? bv.v[e] : st.alpha * bv.v[e];
                const double r64 = bb - wv.v[e];
                const T rt = (T)r64;
                const T zz = pre ? mul_rn(__ldg(irow + axis_class(i0 + e, nx)), rt) : rt;
                rv.v[e] = rt;
                acc[0] += (double)rt * (double)zz;
                acc[1] += (double)rt * (double)rt;
                acc[2] += r64 * r64;
            }
            st4(rdst + g0, rv);
        }
    };

    // ---- Q pass: p = r / diag + beta p_old, A p, p.Ap ------------------------------
    auto qpass = [&](bool first, const T *pold, T *pw, double beta, double &q1) -> bool {
        const CUtensorMap *mp = pold == bufa ? tm_pa : tm_pb;
        const T bt = (T)beta;
        auto issue = [&](const Unit &U, int m, unsigned char *stg, uint64_t *bar) {
            mbar_expect_tx(bar, (unsigned)(L::ELEMS * sizeof(T)) * (first ? 1u : 2u));
            tma_load_3d(stg, tm_r, bar, U.x0 - HX, U.y0 - 1, m);
            if (!first) tma_load_3d(stg + L::ARR, mp, bar, U.x0 - HX, U.y0 - 1, m);
        };
        auto form = [&](const Unit &U, int m, int ts, unsigned char *stg, unsigned char *rp) {
            const T *rs = reinterpret_cast<const T *>(stg);
            const T *itab = tabT(ts) + JOFF;
            const T *ps = reinterpret_cast<const T *>(stg + L::ARR);
            T *dst = reinterpret_cast<T *>(rp);
            const bool own_plane = m >= U.k0 && m < U.k1;
            constexpr int QX = WX / 4;
            for (int e = threadIdx.x; e < L::H * QX; e += blockDim.x) {
                const int h = e / QX, xq = e - h * QX;
                const int o = h * WX + 4 * xq;
                const int i = U.x0 - HX + 4 * xq, j = U.y0 - 1 + h;
                const V4<T> rv = ld4(rs + o);
                V4<T> po = {{T(0), T(0), T(0), T(0)}};
                if (!first) po = ld4(ps + o);
                // away from the x faces the four cells share one class
                const T *irow = itab + axis_class(j, ny) * 3;
                T iv[4];
                if (i > 0 && i + 3 < nx - 1) {
                    iv[0] = iv[1] = iv[2] = iv[3] = irow[1];
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) iv[q] = irow[axis_class(i + q, nx)];
                }
                V4<T> pv;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const T zz = pre ? mul_rn(iv[q], rv.v[q]) : rv.v[q];
                    pv.v[q] = first ? zz : fma(bt, po.v[q], zz);
                }
                st4(dst + o, pv);
                if (own_plane && h >= 1 && h <= W && xq >= HX / 4 && xq < (HX + TX) / 4 && i < nx && j < ny)
                    st4(pw + (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * m), pv);
            }
        };
        auto out = [&](const Unit &U, int k, int ts, unsigned char *lo, unsigned char *mid, unsigned char *hi) {
            const int j = U.y0 + w, i0 = U.x0 + 4 * lane;
            if (j >= ny) return;
            const T *pm = reinterpret_cast<const T *>(mid);
            const V4<T> ap = apply27<T, W>(st, reinterpret_cast<const T *>(lo), pm, reinterpret_cast<const T *>(hi),
                                           tabT(ts), i0, j, w, lane);
            if (i0 >= nx) return;
            const size_t g0 = (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * k);
            st4(apb + g0, ap);
            const V4<T> pc = ld4(pm + (w + 1) * WX + HX + 4 * lane);
#pragma unroll
            for (int e = 0; e < 4; ++e) q1 += (double)pc.v[e] * (double)ap.v[e];
        };
        return zpass<W, S>(z, a, smem, L::TABS, L::STAGE, L::RPLANE, pp, issue, tabs, form, out);
    };

    // ---- window Q pass (QWIN, mixed): the same products without the ring ----------
    // Each warp forms the direction p for its own row and the rows above and
    // below it (one row of four cells per lane) straight from the staged r
    // and p_old, keeps p of the last three planes in registers (win) and
    // applies the stencil from there; stage buffers are handed back per warp
    // through an "empty" mbarrier instead of a block barrier per plane.
    // Entry e of the block's plane sequence (over its units) is staged in
    // stage e % S with r, p_old and the plane's table; its table is read
    // again at entry e + 1 (the product of plane e), so the warp releases
    // stage e at entry e + 1, and thread 0 refills it with entry e + S at
    // entry e + QDLY, after every warp has released it.
    unsigned qbase = 0;    // entries of the earlier window Q passes (mbarrier phases)
    auto qpass_w = [&](bool first, const T *pold, T *pw, double beta, double &q1) -> bool {
        const CUtensorMap *mp = pold == bufa ? tm_pa : tm_pb;
        const T bt = (T)beta;
        uint64_t *full = bars + 4, *empty = bars + 8;
        unsigned char *stage0 = smem + 128 + L::TABS;
        const int units = z.tiles_x * z.tiles_y * z.chunks;
        const unsigned bytes = (unsigned)(L::ELEMS * sizeof(T)) * (first ? 1u : 2u) + (unsigned)(PTAB * 4);
        // producer cursor (thread 0)
        int pun = blockIdx.x, pm = 0;
        Unit PU{0, 0, 0, 0};
        if (pun < units) PU = unit_of<W>(z, nz, pun);
        unsigned issued = 0;
        bool ok = true;
        auto produce = [&]() {
            if (pun >= units || !ok) return;
            const unsigned E = qbase + issued;
            const int s = (int)(E % S);
            if (E >= (unsigned)S && !mbar_wait(&empty[s], (E / S - 1u) & 1u)) {
                ok = false;
                return;
            }
            fence_proxy_async();
            unsigned char *stg = stage0 + (size_t)s * L::STAGE;
            const int m = PU.k0 - 1 + pm;
            const int mc = m < 0 ? 0 : (m >= nz ? nz - 1 : m);
            mbar_expect_tx(&full[s], bytes);
            tma_load_3d(stg, tm_r, &full[s], PU.x0 - HX, PU.y0 - 1, m);
            if (!first) tma_load_3d(stg + L::ARR, mp, &full[s], PU.x0 - HX, PU.y0 - 1, m);
            bulk_load(stg + 2 * L::ARR, z.ptab32 + (size_t)mc * PTAB, (unsigned)(PTAB * 4), &full[s]);
            ++issued;
            if (++pm >= PU.k1 - PU.k0 + 2) {
                pm = 0;
                pun += gridDim.x;
                if (pun < units) PU = unit_of<W>(z, nz, pun);
            }
        };
        if (threadIdx.x == 0)
            for (int i = 0; i < S - QDLY; ++i) produce();
        V4<T> win[3][3];
        T hx[3][3];
#pragma unroll
        for (int pz = 0; pz < 3; ++pz)
#pragma unroll
            for (int ry = 0; ry < 3; ++ry) {
                win[pz][ry] = V4<T>{{T(0), T(0), T(0), T(0)}};
                hx[pz][ry] = T(0);
            }
        unsigned e = 0;       // entries of this pass consumed by this thread
        for (int un = blockIdx.x; un < units && ok; un += gridDim.x) {
            const Unit U = unit_of<W>(z, nz, un);
            const int P = U.k1 - U.k0 + 2;
            const int j = U.y0 + w, i0 = U.x0 + 4 * lane;
            for (int u = 0; u < P; ++u, ++e) {
                const unsigned E = qbase + e;
                const int s = (int)(E % S);
                if (!mbar_wait(&full[s], (E / S) & 1u)) {
                    ok = false;
                    break;
                }
                const unsigned char *stg = stage0 + (size_t)s * L::STAGE;
                const T *rs = reinterpret_cast<const T *>(stg);
                const T *ps = reinterpret_cast<const T *>(stg + L::ARR);
                const float *tb = reinterpret_cast<const float *>(stg + 2 * L::ARR);
                const int m = U.k0 - 1 + u;
#pragma unroll
                for (int ry = 0; ry < 3; ++ry) {
                    win[0][ry] = win[1][ry];
                    win[1][ry] = win[2][ry];
                    hx[0][ry] = hx[1][ry];
                    hx[1][ry] = hx[2][ry];
                }
#pragma unroll
                for (int h = 0; h < 3; ++h) {
                    const int jr = j - 1 + h;
                    const float *irow = tb + JOFF + axis_class(jr, ny) * 3;
                    const int o = (w + h) * WX + HX + 4 * lane;
                    const V4<T> rv = ld4(rs + o);
                    V4<T> po = {{T(0), T(0), T(0), T(0)}};
                    if (!first) po = ld4(ps + o);
                    T iv[4];
                    if (i0 > 0 && i0 + 3 < nx - 1) {
                        iv[0] = iv[1] = iv[2] = iv[3] = (T)irow[1];
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; ++q) iv[q] = (T)irow[axis_class(i0 + q, nx)];
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const T zz = pre ? mul_rn(iv[q], rv.v[q]) : rv.v[q];
                        win[2][h].v[q] = first ? zz : fma(bt, po.v[q], zz);
                    }
                    // the value beyond the tile's edge: left of it in lane 0,
                    // right of it in lane 31 (zero outside the grid)
                    T ph = T(0);
                    if (lane == 0 || lane == 31) {
                        const int ce = lane == 0 ? -1 : 4;
                        const T re = rs[o + ce];
                        const T pe = first ? T(0) : ps[o + ce];
                        const T ie = (T)irow[axis_class(i0 + ce, nx)];
                        const T zz = pre ? mul_rn(ie, re) : re;
                        ph = first ? zz : fma(bt, pe, zz);
                    }
                    hx[2][h] = ph;
                }
                if (m >= U.k0 && m < U.k1 && j < ny && i0 < nx)
                    st4(pw + (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * m), win[2][1]);
                if (u >= 2) {
                    // plane m - 1, with its table (stage of entry e - 1)
                    const float *tp =
                        reinterpret_cast<const float *>(stage0 + (size_t)((E - 1u) % S) * L::STAGE + 2 * L::ARR);
                    const V4<T> ap = apply_w<T>(st, win, hx, tp, i0, j, lane);
                    if (j < ny && i0 < nx) {
                        const size_t g0 = (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * (m - 1));
                        st4(apb + g0, ap);
#pragma unroll
                        for (int q = 0; q < 4; ++q) q1 += (double)win[1][1].v[q] * (double)ap.v[q];
                    }
                }
                // stage of entry e - 1: its table was read for the last time above
                if (e > 0) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[(E - 1u) % S]);
                }
                if (threadIdx.x == 0) produce();
            }
        }
        if (ok && e > 0) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[(qbase + e - 1u) % S]);
        }
        if (!__syncthreads_and(ok)) {
            // let the copies this block started finish before it leaves
            if (threadIdx.x == 0) {
                atomicExch(a.status, MB_ERR_CUDA);
                for (unsigned E = qbase + e; E < qbase + issued; ++E) (void)mbar_wait(&full[E % S], (E / S) & 1u);
            }
            __syncthreads();
            return false;
        }
        qbase += e;
        return true;
    };

    // ---- U pass: x += alpha p, r -= alpha A p; r.z, r.r (z formed, not stored) -----
    auto upass = [&](const T *pc_, double alpha, double (&u2)[2]) {
        const T al = (T)alpha;
        double *__restrict__ x = a.x;
        const unsigned gx = (unsigned)nx >> 2;
        const unsigned groups = gx * (unsigned)ny * (unsigned)nz;
        const unsigned step = gridDim.x * blockDim.x;
        for (unsigned q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < groups; q0 += 2 * step) {
            V4<T> pv[2], av[2], rv[2];
            V4<double> xv[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const unsigned q = q0 + u * step;
                const size_t g0 = (size_t)(q < groups ? q : q0) << 2;
                pv[u] = ld4(pc_ + g0);
                av[u] = ld4(apb + g0);
                rv[u] = ld4(r + g0);
                xv[u] = ld4(x + g0);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const unsigned q = q0 + u * step;
                if (q >= groups) continue;
                const size_t g0 = (size_t)q << 2;
                const unsigned t = z.by_gx.div(q);
                const int i0 = (int)(q - t * gx) << 2;
                const unsigned kk = z.by_ny.div(t);
                const int k = (int)kk, j = (int)(t - kk * (unsigned)ny);
                // Jacobi values of the group: the row's interior class, and
                // its face classes for the first / last cell of an x-row
                T iv[4] = {T(1), T(1), T(1), T(1)};
                if (pre) {
                    const T *irow = invt + k * 9 + axis_class(j, ny) * 3;
                    const T lo = __ldg(irow), mi = __ldg(irow + 1), hi = __ldg(irow + 2);
                    iv[0] = i0 == 0 ? lo : mi;
                    iv[1] = iv[2] = mi;
                    iv[3] = i0 + 3 == nx - 1 ? hi : mi;
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    xv[u].v[e] += alpha * (double)pv[u].v[e];
                    const T rn = fma(-al, av[u].v[e], rv[u].v[e]);
                    rv[u].v[e] = rn;
                    const T zz = pre ? mul_rn(iv[e], rn) : rn;
                    u2[0] += (double)zz * (double)rn;
                    u2[1] += (double)rn * (double)rn;
                }
                st4(x + g0, xv[u]);
                st4(r + g0, rv[u]);
            }
        }
    };

    // ---- fused pass (FUSED, mixed): one stencil pass per iteration -------------
    // Iteration k forms, from the staged r_{k-1}, A p_{k-1} and p_{k-1} (halo
    // included),
    //   r_k = r_{k-1} - alpha_{k-1} A p_{k-1}   (the U pass's FP32 fma)
    //   p_k = r_k / diag + beta_{k-1} p_{k-1}    (the Q pass's)
    // into the ring (p, then r), stores the tile's cells of r_k and p_k,
    // applies x += alx p_{k-1} to the tile's cells (FP64; x of the next plane
    // is loaded one plane ahead), and sums q = A p_k into the partials
    //   p.q, q.z, q.Mq, q.r, q.q, r.z, r.r     (z = M r_k, M = 1 / diag)
    // One reduction then gives r_k.z_k and r_k.r_k of the stored r_k,
    // alpha_k = r.z / p.q, and r_{k+1}.z_{k+1} and r_{k+1}.r_{k+1} as
    //   r.z - 2 a q.z + a^2 q.Mq,   r.r - 2 a q.r + a^2 q.q
    // with a = alpha_k rounded to FP32 (the value the FP32 update of r
    // applies): exact up to the rounding of r_{k+1} itself (about 1e-7
    // relative), which is all beta_k (p_{k+1} is formed before r_{k+1}.z_{k+1}
    // can be summed) and the refinement test need; alpha_{k+1} then uses the
    // stored r_{k+1}'s own sums, so no error accumulates.  r and A p
    // alternate between two buffers, since other blocks read the halo of the
    // ones this pass replaces.  first: r_k is the staged residual and
    // p_k = M r_k (no A p staged); xupd: p_{k-1} is staged for the pending
    // update of x.
    // (selected, not indexed: a run-time index would put the pairs in local memory)
    T *const rb0 = r, *const rb1 = MIXED ? (T *)a.z32 : r;
    T *const ab0 = apb, *const ab1 = MIXED ? (T *)a.ap32b : apb;
    auto rbuf = [&](int i) { return i ? rb1 : rb0; };
    auto fpass = [&](bool first, bool xupd, double alx, int rsel, int asel, const T *pold, T *pw, double alpha,
                     double beta, double (&d7)[7]) -> bool {
        const CUtensorMap *mr = rsel ? z.maps + 4 : tm_r;
        const CUtensorMap *ma = asel ? z.maps + 6 : z.maps + 5;
        const CUtensorMap *mp = pold == bufa ? tm_pa : tm_pb;
        T *rout = rsel ? rb0 : rb1;
        T *aout = asel ? ab0 : ab1;
        const T al = (T)alpha, bt = (T)beta;
        const bool cont = !first;
        const unsigned arrays = 1u + (cont ? 1u : 0u) + ((cont || xupd) ? 1u : 0u);
        auto issue = [&](const Unit &U, int m, unsigned char *stg, uint64_t *bar) {
            mbar_expect_tx(bar, (unsigned)(L::ELEMS * sizeof(T)) * arrays);
            tma_load_3d(stg, mr, bar, U.x0 - HX, U.y0 - 1, m);
            if (cont) tma_load_3d(stg + L::ARR, ma, bar, U.x0 - HX, U.y0 - 1, m);
            if (cont || xupd) tma_load_3d(stg + 2 * L::ARR, mp, bar, U.x0 - HX, U.y0 - 1, m);
        };
        // the lane's four cells of tile row w (x of the plane being updated)
        const int jw = w, xl = 4 * lane;
        V4<double> xnext = {{0.0, 0.0, 0.0, 0.0}};
        auto form = [&](const Unit &U, int m, int ts, unsigned char *stg, unsigned char *rp) {
            const T *rs = reinterpret_cast<const T *>(stg);
            const T *as = reinterpret_cast<const T *>(stg + L::ARR);
            const T *ps = reinterpret_cast<const T *>(stg + 2 * L::ARR);
            const T *itab = tabT(ts) + JOFF;
            T *dp = reinterpret_cast<T *>(rp);
            T *dr = reinterpret_cast<T *>(rp + L::ARR);
            const bool own_plane = m >= U.k0 && m < U.k1;
            constexpr int QX = WX / 4;
            for (int e = threadIdx.x; e < L::H * QX; e += blockDim.x) {
                const int h = e / QX, xq = e - h * QX;
                const int o = h * WX + 4 * xq;
                const int i = U.x0 - HX + 4 * xq, j = U.y0 - 1 + h;
                V4<T> rk = ld4(rs + o);
                V4<T> po = {{T(0), T(0), T(0), T(0)}};
                if (cont) {
                    const V4<T> av = ld4(as + o);
                    po = ld4(ps + o);
#pragma unroll
                    for (int q = 0; q < 4; ++q) rk.v[q] = fma(-al, av.v[q], rk.v[q]);
                }
                const T *irow = itab + axis_class(j, ny) * 3;
                T iv[4];
                if (i > 0 && i + 3 < nx - 1) {
                    iv[0] = iv[1] = iv[2] = iv[3] = irow[1];
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) iv[q] = irow[axis_class(i + q, nx)];
                }
                V4<T> pv;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const T zz = pre ? mul_rn(iv[q], rk.v[q]) : rk.v[q];
                    pv.v[q] = cont ? fma(bt, po.v[q], zz) : zz;
                }
                st4(dp + o, pv);
                st4(dr + o, rk);
                if (own_plane && h >= 1 && h <= W && xq >= HX / 4 && xq < (HX + TX) / 4 && i < nx && j < ny) {
                    const size_t g = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * m);
                    st4(pw + g, pv);
                    if (cont) st4(rout + g, rk);
                }
            }
            if (!xupd) return;
            const int j = U.y0 + jw, i0 = U.x0 + xl;
            if (j >= ny || i0 >= nx) return;
            if (own_plane) {
                const V4<T> pk = ld4(ps + (jw + 1) * WX + HX + xl);
                V4<double> xn;
#pragma unroll
                for (int q = 0; q < 4; ++q) xn.v[q] = fma(alx, (double)pk.v[q], xnext.v[q]);
                st4(a.x + (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * m), xn);
            }
            // x of the next plane of this unit, used by the next step's form
            if (m + 1 >= U.k0 && m + 1 < U.k1)
                xnext = ld4(a.x + (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * (m + 1)));
        };
        auto out = [&](const Unit &U, int k, int ts, unsigned char *lo, unsigned char *mid, unsigned char *hi) {
            const int j = U.y0 + w, i0 = U.x0 + 4 * lane;
            if (j >= ny) return;
            const T *pm = reinterpret_cast<const T *>(mid);
            const V4<T> q = apply27<T, W>(st, reinterpret_cast<const T *>(lo), pm, reinterpret_cast<const T *>(hi),
                                          tabT(ts), i0, j, w, lane);
            if (i0 >= nx) return;
            const size_t g0 = (size_t)i0 + (size_t)nx * ((size_t)j + (size_t)ny * k);
            st4(aout + g0, q);
            const int oc = (w + 1) * WX + HX + 4 * lane;
            const V4<T> pc = ld4(pm + oc);
            const V4<T> rc = ld4(reinterpret_cast<const T *>(mid + L::ARR) + oc);
            T iv[4] = {T(1), T(1), T(1), T(1)};
            if (pre) {
                const T *irow = tabT(ts) + JOFF + axis_class(j, ny) * 3;
                iv[0] = i0 == 0 ? irow[0] : irow[1];
                iv[1] = iv[2] = irow[1];
                iv[3] = i0 + 3 == nx - 1 ? irow[2] : irow[1];
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const double qd = (double)q.v[e];
                const T zz = pre ? mul_rn(iv[e], rc.v[e]) : rc.v[e];
                const T mq = pre ? mul_rn(iv[e], q.v[e]) : q.v[e];
                const double rd = (double)rc.v[e];
                d7[0] += (double)pc.v[e] * qd;
                d7[1] += qd * (double)zz;
                d7[2] += qd * (double)mq;
                d7[3] += qd * rd;
                d7[4] += qd * qd;
                d7[5] += rd * (double)zz;
                d7[6] += rd * rd;
            }
        };
        return zpass<W, S>(z, a, smem, L::TABS, L::STAGE, L::RPLANE, pp, issue, tabs, form, out);
    };

    if constexpr (MODE == FUSED) {
        // The mixed loop of the other forms (same refinement rule and stop
        // test), with one reduction per iteration.  x of the last direction
        // is applied by the next fused pass, or by the residual pass's input
        // and then the final sweep below.
        double acc[3] = {0.0, 0.0, 0.0}, s3[3];
        const bool wv = a.w != nullptr && c->w_valid != 0;
        if (wv) residual_w(rbuf(0), acc);
        else if (!residual(rbuf(0), nullptr, 0.0, acc)) return;
        if (!grid_reduce<3, 32 * W>(a, acc, s3, red)) return;
        if (wv && !(s3[2] >= tol)) {
            // the solve would stop here: decide on the stencil's residual
            double t3[3] = {0.0, 0.0, 0.0};
            if (!residual(rbuf(0), nullptr, 0.0, t3)) return;
            if (!grid_reduce<3, 32 * W>(a, t3, s3, red)) return;
        }
        double rz = s3[0], rr = s3[1];
        double error = s3[2], rr_ref = s3[2];
        int its = 1, refinements = 1;
        bool done = !(s3[2] >= tol) || !(1 < max_its);
        bool first = true, xupd = false;
        double alpha = 0.0, beta = 0.0;
        int rsel = 0, asel = 0;
        T *pcur = bufb;
        while (!done) {
            T *pnew = pcur == bufa ? bufb : bufa;
            double d7[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, s7[7];
            if (!fpass(first, xupd, alpha, rsel, asel, pcur, pnew, alpha, beta, d7)) return;
            if (!grid_reduce<7, 32 * W>(a, d7, s7, red)) return;
            if (!first) rsel ^= 1;
            asel ^= 1;
            pcur = pnew;
            rz = s7[5];
            rr = s7[6];
            alpha = (pre ? rz : rr) / s7[0];
            const double af = (double)(T)alpha;
            const double rz_n = rz - 2.0 * af * s7[1] + af * af * s7[2];
            const double rr_n = rr - 2.0 * af * s7[3] + af * af * s7[4];
            xupd = true;
            its += 1;
            if (rr_n <= fmax(c->refine_floor, ratio * rr_ref) || its >= max_its) {
                double t3[3] = {0.0, 0.0, 0.0};
                if (!residual(rbuf(rsel), pcur, alpha, t3)) return;
                if (!grid_reduce<3, 32 * W>(a, t3, s3, red)) return;
                refinements += 1;
                error = s3[2];
                rr_ref = s3[2];
                rz = s3[0];
                rr = s3[1];
                first = true;
                if (s3[2] <= tol || its >= max_its) done = true;
            } else {
                beta = pre ? rz_n / rz : rr_n / rr;
                rz = rz_n;
                rr = rr_n;
                error = rr_n;
                first = false;
            }
        }
        if (xupd) {
            // x += alpha p of the last direction; every block has finished the
            // residual pass that read x (its reduction was a grid barrier)
            const unsigned groups = (unsigned)(nx >> 2) * (unsigned)ny * (unsigned)nz;
            for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < groups; q += gridDim.x * blockDim.x) {
                const size_t g0 = (size_t)q << 2;
                const V4<T> pv = ld4(pcur + g0);
                V4<double> xv = ld4(a.x + g0);
#pragma unroll
                for (int e = 0; e < 4; ++e) xv.v[e] = fma(alpha, (double)pv.v[e], xv.v[e]);
                st4(a.x + g0, xv);
            }
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            c->its = its;
            c->error = error;
            c->refinements = refinements;
            c->rz = rz;
            c->rr = rr;
            // w is A x of the solution when a refinement residual formed it, or
            // when it was valid and x did not move
            c->w_valid = (a.w != nullptr && (refinements > 1 || wv)) ? 1 : 0;
            c->done = 1;
        }
        return;
    }

    double acc[3] = {0.0, 0.0, 0.0}, s3[3];
    if (!residual(r, nullptr, 0.0, acc)) return;
    if (!grid_reduce<3, 32 * W>(a, acc, s3, red)) return;
    double rz = s3[0], rr = s3[1];
    double error = s3[2], rr_ref = s3[2];
    int its = 1, refinements = MIXED ? 1 : 0;
    bool done = !(s3[2] >= tol) || !(1 < max_its);
    bool first = true;
    double beta = 0.0;
    T *pcur = bufb;

    while (!done) {
        T *pnew = pcur == bufa ? bufb : bufa;
        double q1[1] = {0.0}, s1[1];
        bool qok;
        if constexpr (MODE == QWIN && MIXED) qok = qpass_w(first, pcur, pnew, beta, q1[0]);
        else qok = qpass(first, pcur, pnew, beta, q1[0]);
        if (!qok) return;
        if (!grid_reduce<1, 32 * W>(a, q1, s1, red)) return;
        const double alpha = (pre ? rz : rr) / s1[0];
        pcur = pnew;

        double u2[2] = {0.0, 0.0}, s2[2];
        upass(pcur, alpha, u2);
        if (!grid_reduce<2, 32 * W>(a, u2, s2, red)) return;
        its += 1;
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
                if (!residual(r, nullptr, 0.0, t3)) return;
                if (!grid_reduce<3, 32 * W>(a, t3, s3, red)) return;
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
        c->w_valid = 0;          // x moved without the fused solve's product
        c->done = 1;
    }
}

// Jacobi 1/diag per plane and row class: 1 / the class row's diagonal entry;
// and the padded FP32 per-plane blocks of the window Q pass (class rows,
// Jacobi values, zeros).
__global__ void k_zinv(mb_stencil_dev st, double *inv64, float *inv32, float *ptab32) {
    const int n = st.nz * 9;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        inv64[e] = 1.0 / st.table[(size_t)e * 27 + 13];
        inv32[e] = 1.0f / (st.table32 ? st.table32[(size_t)e * 27 + 13] : (float)st.table[(size_t)e * 27 + 13]);
    }
    if (!ptab32) return;
    const int np = st.nz * PTAB;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < np; e += gridDim.x * blockDim.x) {
        const int k = e / PTAB, q = e - k * PTAB;
        float v = 0.0f;
        if (q < JOFF) {
            const int row = q / CROW, col = q - row * CROW;
            if (col < 27) {
                const size_t src = (size_t)k * 243 + row * 27 + col;
                v = st.table32 ? st.table32[src] : (float)st.table[src];
            }
        } else if (q < JOFF + 9) {
            const size_t src = ((size_t)k * 9 + (q - JOFF)) * 27 + 13;
            v = 1.0f / (st.table32 ? st.table32[src] : (float)st.table[src]);
        }
        ptab32[e] = v;
    }
}

// ---- variants ---------------------------------------------------------------------

struct Variant {
    const void *fn;
    int warps;     // tile rows W (threads = 32 W)
    int bytes;     // dynamic shared memory
    int mode;      // QRING, QWIN or FUSED
};

template <bool MIXED, int W, int S, int MINB, int MODE = QRING>
constexpr Variant make() {
    return {(const void *)k_zcg<MIXED, W, S, MINB, MODE>, W, Lay<typename Prec<MIXED>::T, W, S, MODE>::BYTES, MODE};
}

// Mixed: 4-6 run the window Q pass, 7-9 the fused pass.  FP64 has neither
// (its iterations keep the U pass, whose r.r decides the stop exactly as the
// reference's loop does); its 4-6 are ring-pass shapes whose shared memory
// fits (four stages of FP64 planes of W = 16 do not) and 7-9 are empty.
constexpr int NUM_VARIANTS = 10;

static Variant variant(int mixed, int v) {
    static const Variant t64[NUM_VARIANTS] = {make<false, 8, 3, 1>(),  make<false, 8, 3, 2>(),
                                              make<false, 16, 3, 1>(), make<false, 4, 3, 3>(),
                                              make<false, 8, 4, 2>(),  make<false, 16, 3, 1>(),
                                              make<false, 4, 4, 3>(),  Variant{nullptr, 0, 0, 0},
                                              Variant{nullptr, 0, 0, 0},  Variant{nullptr, 0, 0, 0}};
    static const Variant t32[NUM_VARIANTS] = {
        make<true, 8, 3, 1>(),        make<true, 8, 3, 2>(),         make<true, 16, 3, 1>(),
        make<true, 4, 3, 3>(),        make<true, 8, 4, 2, QWIN>(),   make<true, 16, 4, 1, QWIN>(),
        make<true, 4, 4, 3, QWIN>(),  make<true, 8, 3, 2, FUSED>(),  make<true, 16, 3, 1, FUSED>(),
        make<true, 4, 3, 3, FUSED>()};
    return mixed ? t32[v] : t64[v];
}

// Resident blocks of a variant per SM x SMs (0 where it does not fit).
static int grid_of(const Variant &var) {
    if (!var.fn) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(var.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, var.bytes) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, var.fn, 32 * var.warps, var.bytes) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return sms * per;
}

// The multiply-shift constants of FastDiv for divisor d >= 1.
static FastDiv fastdiv(uint32_t d) {
    FastDiv f{d, 0u, 0u};
    if (d > 1) {
        uint32_t l = 0;
        while ((1ull << l) < d) ++l;
        f.l = l;
        f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    }
    return f;
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiled encoder() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        fn = (EncodeTiled)p;
    }
    return fn;
}

// A 3-D map of an nx x ny x nz grid vector with a box of WX x (W + 2) x 1
// cells; reads outside the grid return zeros.
static int encode(CUtensorMap *m, const void *base, int elem, int nx, int ny, int nz, int W) {
    EncodeTiled fn = encoder();
    if (!fn || !base) return 0;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * elem, (cuuint64_t)nx * ny * elem};
    const cuuint32_t box[3] = {(cuuint32_t)WX, (cuuint32_t)(W + 2), 1};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = fn(m, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                          const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace zcg
}  // namespace mb

using namespace mb::zcg;

extern "C" int mbk_zcg_variants(void) { return NUM_VARIANTS; }

// Grid size of variant v (blocks resident at once), 0 if it cannot run.
extern "C" int mbk_zcg_max_blocks(int mixed, int v) {
    if (v < 0 || v >= NUM_VARIANTS) return 0;
    return grid_of(variant(mixed, v));
}

// Whether the z-march kernel applies: the 27-point class-table operator on a
// grid whose rows are whole 16-byte vectors (nx % 4 == 0).
extern "C" int mbk_zcg_usable(const mb_stencil_dev *st) {
    return st->kind == 2 && st->nx % 4 == 0 && st->nx >= 8 && st->ny >= 1 && st->nz >= 1 && st->table &&
           st->table32;
}

// Per-plane Jacobi tables (device arrays of nz * 9 values each) and the
// padded per-plane blocks (nz * PTAB floats; may be NULL).
extern "C" int mbk_zcg_inv_tables(const mb_stencil_dev *st, double *inv64, float *inv32, float *ptab32,
                                  cudaStream_t s) {
    k_zinv<<<(st->nz * PTAB + 255) / 256, 256, 0, s>>>(*st, inv64, inv32, ptab32);
    return (int)cudaGetLastError();
}

extern "C" int mbk_zcg_ptab_floats(void) { return PTAB; }

// Tensor maps of every variant (MAPS per variant: r, p buffer a, p buffer b,
// x, and for the fused pass the second r buffer and both A p buffers),
// encoded on the host and copied to a device array p->zc_maps allocated here
// (freed by the tissue).  Called once the CG buffers exist, before any
// launch or stream capture.  Returns 0 or a CUDA error code.
extern "C" int mbk_zcg_prepare(mb_pcg_dev *p) {
    const int nx = p->st.nx, ny = p->st.ny, nz = p->st.nz;
    const int elem = p->mixed ? 4 : 8;
    alignas(64) CUtensorMap tm[NUM_VARIANTS * MAPS];
    memset(tm, 0, sizeof tm);
    const void *bases[MAPS] = {p->mixed ? (const void *)p->r32 : (const void *)p->r64,
                               p->mixed ? (const void *)p->pa32 : (const void *)p->pa64,
                               p->mixed ? (const void *)p->pb32 : (const void *)p->pb64,
                               (const void *)p->x,
                               p->mixed ? (const void *)p->z32 : nullptr,
                               p->mixed ? (const void *)p->ap32 : nullptr,
                               p->mixed ? (const void *)p->ap32b : nullptr,
                               nullptr};
    for (int v = 0; v < NUM_VARIANTS; ++v) {
        const Variant var = variant(p->mixed, v);
        if (!var.fn) continue;
        for (int q = 0; q < MAPS; ++q) {
            // the fused pass's extra maps exist where its buffers do
            if (q >= 4 && !bases[q]) continue;
            if (!encode(&tm[MAPS * v + q], bases[q], q == 3 ? 8 : elem, nx, ny, nz, var.warps))
                return (int)cudaErrorInvalidValue;
        }
    }
    if (!p->zc_maps) {
        cudaError_t e = cudaMalloc(&p->zc_maps, sizeof tm);
        if (e != cudaSuccess) return (int)e;
    }
    return (int)cudaMemcpy(p->zc_maps, tm, sizeof tm, cudaMemcpyHostToDevice);
}

extern "C" int mbk_zcg_launch(const mb_pcg_dev *p, cudaStream_t s) {
    if (p->zc_variant < 0 || p->zc_variant >= NUM_VARIANTS || !p->zc_maps) return (int)cudaErrorInvalidValue;
    const Variant var = variant(p->mixed, p->zc_variant);
    if (!var.fn) return (int)cudaErrorInvalidValue;
    // the fused pass alternates r and A p between two buffers each
    if (var.mode == FUSED && (!p->z32 || !p->ap32b)) return (int)cudaErrorInvalidValue;
    const int nx = p->st.nx, ny = p->st.ny, nz = p->st.nz;
    const int blocks = p->blocks;
    if (blocks <= 0) return (int)cudaErrorInvalidConfiguration;
    // units: x tiles of 128 cells, y tiles of W rows, z chunks; the number of
    // chunks minimises the rounds of units the grid takes times the planes a
    // unit walks (its planes plus the two halo planes)
    ZArgs z;
    z.inv64 = p->zc_inv64;
    z.inv32 = p->zc_inv32;
    z.ptab32 = p->zc_ptab32;
    z.maps = reinterpret_cast<const CUtensorMap *>(p->zc_maps) + MAPS * p->zc_variant;
    z.tiles_x = (nx + TX - 1) / TX;
    z.tiles_y = (ny + var.warps - 1) / var.warps;
    z.by_gx = fastdiv((uint32_t)(nx / 4));
    z.by_ny = fastdiv((uint32_t)ny);
    {
        long long best = -1;
        int bc = 1;
        for (int c = 1; c <= nz && c <= 64; ++c) {
            const long long units = (long long)z.tiles_x * z.tiles_y * c;
            const long long rounds = (units + blocks - 1) / blocks;
            const long long cost = rounds * ((nz + c - 1) / c + 2);
            if (best < 0 || cost < best) {
                best = cost;
                bc = c;
            }
        }
        z.chunks = bc;
        // balanced ranges: planes per block plus two halo planes for each
        // tile a range can touch; the window Q pass walks units only.
        // MB_ZCG_SCHEDULE=chunks|balanced overrides the choice (tuning).
        const long long pairs = (long long)z.tiles_x * z.tiles_y * nz;
        const long long per = (pairs + blocks - 1) / blocks;
        const long long bal = per + 2 * ((per + nz - 1) / nz + 1);
        z.balanced = var.mode != QWIN && bal < best;
        const char *env = getenv("MB_ZCG_SCHEDULE");
        if (env && var.mode != QWIN) {
            if (!strcmp(env, "chunks")) z.balanced = 0;
            else if (!strcmp(env, "balanced")) z.balanced = 1;
        }
    }
    Args a;
    a.st = p->st;
    a.x = p->x; a.vstar = p->vstar; a.b = p->b;
    a.r64 = p->r64; a.pa64 = p->pa64; a.pb64 = p->pb64; a.z64 = p->z64;
    a.r32 = p->r32; a.pa32 = p->pa32; a.pb32 = p->pb32; a.z32 = p->z32;
    a.ap64 = p->ap64; a.ap32 = p->ap32; a.ap32b = p->ap32b;
    a.w = var.mode == FUSED ? p->zc_w : nullptr;
    {
        // MB_ZCG_STORED_PRODUCT=0: every solve starts with the stencil residual (tuning)
        const char *env = getenv("MB_ZCG_STORED_PRODUCT");
        if (env && !strcmp(env, "0")) a.w = nullptr;
    }
    a.inv_diag64 = p->inv_diag64; a.inv_diag32 = p->inv_diag32;
    a.partials = p->partials; a.ctrl = p->ctrl; a.bar = p->bar; a.status = p->status;
    cudaError_t e = cudaMemsetAsync(p->bar, 0, 2 * sizeof(unsigned), s);
    if (e != cudaSuccess) return (int)e;
    void *args[] = {&a, &z};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(32 * var.warps);
    cfg.dynamicSmemBytes = var.bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelExC(&cfg, var.fn, args);
}

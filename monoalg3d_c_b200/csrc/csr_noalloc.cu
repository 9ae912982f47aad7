// Allocation-free variant of the general CSR conjugate gradient
// (mb_csr_conjugate_gradient).
//
// Who needs it: code that must not allocate device memory while it runs --
// for example a caller working inside a memory budget fixed by its host
// framework (its own pool owns every byte, and a cudaMalloc there would either
// fail or fragment it), a real-time loop in which cudaMalloc's implicit device
// synchronisation and unpredictable latency are not acceptable, or a plugin
// that is handed device buffers by a host application and has no allocator of
// its own.  Such a caller passes its matrix, right-hand side and solution
// already in device memory; this entry point uses no cudaMalloc, cudaFree or
// allocating library routine.
//
// Its work vectors (r, p, q, 1/diag), the block partial sums and the CG control
// block live in one file-scope device array, mb_noalloc_scratch, of
// MB_NOALLOC_SCRATCH_BYTES (16 MiB + 64 KiB).  Every GPU that loads this library
// holds that array until the process exits; under CUDA's lazy module loading
// the array (and the module) are placed on a device at the first call made
// there, which may synchronise the device -- a caller with a fixed budget or
// a real-time loop makes one warm-up call at initialisation.  The device
// address of the array is obtained once per device with
// cudaGetSymbolAddress, on that first call; make it before any stream
// capture on the device.  Each call waits on its stream while it runs (it
// reads the convergence flag back to the host), and the stream must belong
// to the current device.  All calls share the array and it keeps the last
// call's contents: each call rewrites the control block (the only part that
// must start from known values) before launching, and every vector is written
// before it is read.  Calls whose work overlaps on the GPU -- on two streams,
// or from two host threads -- race on the array and must be serialised by the
// caller.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>
#include "mb_internal.h"

// Largest system: the four work vectors of n doubles must fit after the
// control block and the partial sums.
#define MB_NOALLOC_MAX_ROWS (1 << 19)
#define MB_NOALLOC_HEADER_BYTES (64 * 1024)
#define MB_NOALLOC_SCRATCH_BYTES ((size_t)MB_NOALLOC_HEADER_BYTES + 4ull * MB_NOALLOC_MAX_ROWS * sizeof(double))

static __device__ __align__(256) unsigned char mb_noalloc_scratch[MB_NOALLOC_SCRATCH_BYTES];

static_assert(sizeof(mb_ctrl) <= 4096, "the control block must fit before the partial sums");

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char *g_scratch[kMaxDevices];   // device address of the array, per device

// Device address of the scratch array on the current device, looked up once.
int scratch_for_current_device(unsigned char **out, char *err, size_t errlen) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        snprintf(err, errlen, "cudaGetDevice failed: %s", cudaGetErrorString(e));
        return MB_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        snprintf(err, errlen, "device ordinal %d out of range", dev);
        return MB_ERR_ARG;
    }
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, mb_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            snprintf(err, errlen, "cudaGetSymbolAddress(mb_noalloc_scratch) failed on device %d: %s", dev,
                     cudaGetErrorString(e));
            return MB_ERR_CUDA;
        }
        g_scratch[dev] = (unsigned char *)p;
    }
    *out = g_scratch[dev];
    return MB_OK;
}

}  // namespace

extern "C" int mb_noalloc_set_error(int code, const char *msg);

extern "C" int mb_csr_conjugate_gradient_noalloc(int32_t n, const int32_t *row_ptr, const int32_t *col,
                                                 const double *val, const double *b, double *x,
                                                 double tolerance, int max_iterations, int use_preconditioner,
                                                 uint32_t *number_of_iterations, double *error, void *stream) {
    char err[256];
    if (n <= 0 || !row_ptr || !col || !val || !b || !x)
        return mb_noalloc_set_error(MB_ERR_ARG, "mb_csr_conjugate_gradient_noalloc: bad arguments");
    if (n > MB_NOALLOC_MAX_ROWS) {
        snprintf(err, sizeof err,
                 "mb_csr_conjugate_gradient_noalloc: n = %d rows exceeds the allocation-free limit of %d rows",
                 (int)n, (int)MB_NOALLOC_MAX_ROWS);
        return mb_noalloc_set_error(MB_ERR_ARG, err);
    }
    unsigned char *base = nullptr;
    int rc = scratch_for_current_device(&base, err, sizeof err);
    if (rc) return mb_noalloc_set_error(rc, err);
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        int sdev = -1, cur = -1;
        if (cudaStreamGetDevice(s, &sdev) != cudaSuccess || cudaGetDevice(&cur) != cudaSuccess || sdev != cur) {
            cudaGetLastError();
            return mb_noalloc_set_error(MB_ERR_ARG, "mb_csr_conjugate_gradient_noalloc: the stream does not "
                                                    "belong to the current device");
        }
    }

    // layout: [control block][partials][r][p][q][1/diag]
    int gb = (n + 255) / 256;
    if (gb > mbk_max_grid_blocks()) gb = mbk_max_grid_blocks();
    if ((size_t)gb * 3 * sizeof(double) > MB_NOALLOC_HEADER_BYTES - 4096)
        return mb_noalloc_set_error(MB_ERR_ARG, "mb_csr_conjugate_gradient_noalloc: partial sums exceed the header");
    mb_ctrl *ctrl = (mb_ctrl *)base;
    double *partials = (double *)(base + 4096);
    double *vec = (double *)(base + MB_NOALLOC_HEADER_BYTES);
    mb_csr_dev a;
    memset(&a, 0, sizeof a);
    a.n = n;
    a.row_ptr = row_ptr;
    a.col = col;
    a.val = val;
    a.b = b;
    a.x = x;
    a.r = vec;
    a.p = vec + (size_t)n;
    a.q = vec + 2 * (size_t)n;
    a.inv_diag = vec + 3 * (size_t)n;
    a.partials = partials;
    a.grid_blocks = gb;

    mb_ctrl c;
    memset(&c, 0, sizeof c);
    c.tol = tolerance;
    c.max_its = max_iterations;
    c.use_precond = use_preconditioner ? 1 : 0;
    cudaError_t e = cudaMemcpyAsync(ctrl, &c, sizeof c, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        snprintf(err, sizeof err, "control block upload failed: %s", cudaGetErrorString(e));
        return mb_noalloc_set_error(MB_ERR_CUDA, err);
    }
    if (mbk_csr_cg_init(&a, ctrl, s)) return mb_noalloc_set_error(MB_ERR_CUDA, "CSR CG initial launch failed");
    for (int it = 0; it < max_iterations + 1; it += 16) {
        for (int q = 0; q < 16; ++q)
            if (mbk_csr_cg_iter(&a, ctrl, s)) return mb_noalloc_set_error(MB_ERR_CUDA, "CSR CG launch failed");
        int32_t done = 0;
        e = cudaMemcpyAsync(&done, &ctrl->done, sizeof done, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            snprintf(err, sizeof err, "CSR CG failed: %s", cudaGetErrorString(e));
            return mb_noalloc_set_error(MB_ERR_CUDA, err);
        }
        if (done) break;
    }
    e = cudaMemcpyAsync(&c, ctrl, sizeof c, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        snprintf(err, sizeof err, "CSR CG result read failed: %s", cudaGetErrorString(e));
        return mb_noalloc_set_error(MB_ERR_CUDA, err);
    }
    if (number_of_iterations) *number_of_iterations = (uint32_t)c.its;
    if (error) *error = c.error;
    return MB_OK;
}

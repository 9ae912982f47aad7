/* Host driver of the B200 monodomain step (C).
 *
 * Owns the device buffers of one tissue, assembles the diffusion operator,
 * builds the per-step CUDA graph
 *
 *     [ ODE kernel -> CG initial residual ] -> WHILE(cond){ CG iteration } -> [ clock ]
 *
 * and exposes the reference's plugin entry points through the C ABI of
 * include/monoalg3d_b200.h.  Everything in the timed loop runs on the device;
 * the host only launches graphs.
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "mb_internal.h"
#include "mb_assembly.h"
#include "mb_tissue.h"

/* ---- error reporting ----------------------------------------------------- */

static __thread char g_err[512];

static int set_err(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

const char *mb_last_error(void) { return g_err; }

/* Error reporting for the allocation-free entry point (csr_noalloc.cu). */
int mb_noalloc_set_error(int code, const char *msg) { return set_err(code, "%s", msg); }
int mb_version(void) { return 10000; }

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_err(MB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                           __FILE__, __LINE__);                                            \
    } while (0)

#define CKK(call)                                                                          \
    do {                                                                                   \
        int e_ = (call);                                                                   \
        if (e_ != 0)                                                                       \
            return set_err(MB_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                    \
                           cudaGetErrorString((cudaError_t)e_), __FILE__, __LINE__);       \
    } while (0)

int mb_device_count(int *count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    *count = n;
    return MB_OK;
}

/* ---- model tables -------------------------------------------------------- */

int mb_init_cell_model_data(int model, int *neq, double *initial_v) {
    if (model == MB_MODEL_TT2006) {
        if (neq) *neq = MB_NEQ_TT2006;
        if (initial_v) *initial_v = (double)-85.23f;          /* INITIAL_V, ten_tusscher_2006.h:7 */
        return MB_OK;
    }
    if (model == MB_MODEL_TORORD_FKATP_MIXED) {
        if (neq) *neq = MB_NEQ_TORORD;
        if (initial_v) *initial_v = -88.763800;               /* ToRORd_fkatp_mixed_endo_mid_epi.h:11 */
        return MB_OK;
    }
    if (model == MB_MODEL_TORORD_FKATP_ENDO) {
        if (neq) *neq = MB_NEQ_TORORD;
        if (initial_v) *initial_v = (double)-88.763800f;      /* ToRORd_fkatp_endo.h:5 */
        return MB_OK;
    }
    return set_err(MB_ERR_ARG, "unknown model %d", model);
}

int mb_torord_endo_initial_state(int gpu_build, double *state) {
    if (!state) return set_err(MB_ERR_ARG, "null state");
    for (int s = 0; s < MB_NEQ_TORORD; ++s) state[s] = mb_torord_endo_default_state(gpu_build, s);
    return MB_OK;
}

int mb_torord_initial_state(int celltype, double *state) {
    if (!state || celltype < 0 || celltype > 2) return set_err(MB_ERR_ARG, "bad arguments");
    for (int s = 0; s < MB_NEQ_TORORD; ++s) state[s] = mb_torord_default_state(celltype, s);
    return MB_OK;
}

/* Row counts of the SoA state for (model, precision, adaptive ODE step). */
static void ode_rows(int model, int precision, int adaptive, int *n64, int *n32) {
    if (model == MB_MODEL_TORORD_FKATP_ENDO) {
        /* FP64 in either precision; adaptive: + dt, time_new, previous_dt */
        *n64 = MB_NEQ_TORORD + (adaptive ? 3 : 0);
        *n32 = 0;
    } else if (model == MB_MODEL_TT2006) {
        if (precision == MB_PREC_FP64) { *n64 = 19; *n32 = 0; }
        else { *n64 = 6; *n32 = 13; }
    } else {
        if (precision == MB_PREC_FP64) { *n64 = 43; *n32 = 0; }
        else { *n64 = 9; *n32 = 34; }
    }
}

static uint32_t round_up32(uint32_t n) { return (n + 31u) & ~31u; }

/* ---- standalone ODE object ---------------------------------------------- */

struct mb_ode {
    mb_ode_dev dev;
    int neq;
    double *d_stim;
    cudaStream_t stream;
};

int mb_ode_create(mb_ode **out, int model, int precision, int rl_rule, uint32_t num_cells, double dt,
                  uint32_t num_steps) {
    if (!out || num_cells == 0 || dt <= 0.0 || num_steps == 0)
        return set_err(MB_ERR_ARG, "mb_ode_create: bad arguments");
    int neq;
    if (mb_init_cell_model_data(model, &neq, NULL)) return MB_ERR_ARG;
    if (precision != MB_PREC_FP64 && precision != MB_PREC_MIXED) return set_err(MB_ERR_ARG, "bad precision");
    mb_ode *o = (mb_ode *)calloc(1, sizeof *o);
    if (!o) return set_err(MB_ERR_NOMEM, "out of host memory");
    o->neq = neq;
    o->dev.model = model;
    o->dev.precision = model == MB_MODEL_TORORD_FKATP_ENDO ? MB_PREC_FP64 : precision;
    o->dev.rl_rule = rl_rule;
    o->dev.num_steps = (int)num_steps;
    o->dev.n = num_cells;
    o->dev.ld = round_up32(num_cells);
    o->dev.dt = dt;
    int n64, n32;
    ode_rows(model, precision, 0, &n64, &n32);
    cudaError_t e = cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void **)&o->dev.sv64, (size_t)n64 * o->dev.ld * sizeof(double));
    if (e == cudaSuccess && n32) e = cudaMalloc((void **)&o->dev.sv32, (size_t)n32 * o->dev.ld * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc((void **)&o->d_stim, (size_t)num_cells * sizeof(double));
    if (e != cudaSuccess) {
        mb_ode_destroy(o);
        return set_err(MB_ERR_CUDA, "mb_ode_create: %s", cudaGetErrorString(e));
    }
    *out = o;
    return MB_OK;
}

void mb_ode_destroy(mb_ode *o) {
    if (!o) return;
    cudaFree(o->dev.sv64);
    cudaFree(o->dev.sv32);
    cudaFree(o->d_stim);
    if (o->stream) cudaStreamDestroy(o->stream);
    free(o);
}

/* Initial-condition table: ntypes rows of neq doubles. */
static int model_ic_table(int model, const double *initial_state, double *table, int *ntypes) {
    if (model == MB_MODEL_TT2006) {
        for (int s = 0; s < MB_NEQ_TT2006; ++s) table[s] = initial_state ? initial_state[s] : mb_tt2006_default_state(s);
        *ntypes = 1;
    } else if (model == MB_MODEL_TORORD_FKATP_ENDO) {
        for (int s = 0; s < MB_NEQ_TORORD; ++s)
            table[s] = initial_state ? initial_state[s] : mb_torord_endo_default_state(0, s);
        *ntypes = 1;
    } else {
        if (initial_state) {
            for (int s = 0; s < MB_NEQ_TORORD; ++s) table[s] = initial_state[s];
            *ntypes = 1;
        } else {
            for (int t = 0; t < 3; ++t)
                for (int s = 0; s < MB_NEQ_TORORD; ++s) table[t * MB_NEQ_TORORD + s] = mb_torord_default_state(t, s);
            *ntypes = 3;
        }
    }
    return MB_OK;
}

int mb_set_model_initial_conditions_gpu(mb_ode *o, const double *initial_state, const uint8_t *celltype,
                                        size_t *pitch_out) {
    if (!o) return set_err(MB_ERR_ARG, "null ode");
    double table[3 * MB_MAX_NEQ];
    int ntypes;
    model_ic_table(o->dev.model, initial_state, table, &ntypes);
    double *d_table = NULL;
    uint8_t *d_ct = NULL;
    CK(cudaMalloc((void **)&d_table, sizeof table));
    CK(cudaMemcpyAsync(d_table, table, sizeof table, cudaMemcpyHostToDevice, o->stream));
    mb_ode_dev dv = o->dev;
    if (celltype && ntypes > 1) {
        CK(cudaMalloc((void **)&d_ct, o->dev.n));
        CK(cudaMemcpyAsync(d_ct, celltype, o->dev.n, cudaMemcpyHostToDevice, o->stream));
        dv.celltype = d_ct;
    }
    CKK(mbk_ode_init(&dv, d_table, ntypes, o->stream));
    CK(cudaStreamSynchronize(o->stream));
    cudaFree(d_table);
    if (d_ct) {
        /* keep the cell types for the solve calls */
        if (o->dev.celltype) cudaFree((void *)o->dev.celltype);
        o->dev.celltype = d_ct;
    }
    if (pitch_out) *pitch_out = (size_t)o->dev.ld * sizeof(double);
    return MB_OK;
}

int mb_solve_model_odes_gpu(mb_ode *o, double current_t, const double *stim_currents) {
    if (!o) return set_err(MB_ERR_ARG, "null ode");
    mb_ode_dev dv = o->dev;
    dv.cur_time = current_t;
    if (stim_currents) {
        CK(cudaMemcpyAsync(o->d_stim, stim_currents, (size_t)o->dev.n * sizeof(double), cudaMemcpyHostToDevice,
                           o->stream));
    } else {
        CK(cudaMemsetAsync(o->d_stim, 0, (size_t)o->dev.n * sizeof(double), o->stream));
    }
    dv.stim_host = o->d_stim;
    /* V lives in row 0 of the double rows: read and written in place */
    CKK(mbk_ode_step(&dv, NULL, dv.sv64, dv.sv64, o->stream));
    CK(cudaStreamSynchronize(o->stream));
    return MB_OK;
}

int mb_ode_get_state(mb_ode *o, double *host_state) {
    if (!o || !host_state) return set_err(MB_ERR_ARG, "null argument");
    double *d = NULL;
    const size_t bytes = (size_t)o->neq * o->dev.n * sizeof(double);
    CK(cudaMalloc((void **)&d, bytes));
    CKK(mbk_ode_gather(&o->dev, NULL, d, o->stream));
    CK(cudaMemcpyAsync(host_state, d, bytes, cudaMemcpyDeviceToHost, o->stream));
    CK(cudaStreamSynchronize(o->stream));
    cudaFree(d);
    return MB_OK;
}

int mb_ode_set_state(mb_ode *o, const double *host_state) {
    if (!o || !host_state) return set_err(MB_ERR_ARG, "null argument");
    double *d = NULL;
    const size_t bytes = (size_t)o->neq * o->dev.n * sizeof(double);
    CK(cudaMalloc((void **)&d, bytes));
    CK(cudaMemcpyAsync(d, host_state, bytes, cudaMemcpyHostToDevice, o->stream));
    CKK(mbk_ode_scatter(&o->dev, d, NULL, o->stream));
    CK(cudaStreamSynchronize(o->stream));
    cudaFree(d);
    return MB_OK;
}

/* V of every cell (row 0 of the state) from / to host memory with an
 * element stride: stride = the number of equations reads and writes the
 * reference's array-of-structures state vector (sv[i * neq]) in place. */
int mb_ode_device_state(mb_ode *o, double **sv, size_t *pitch) {
    if (!o) return set_err(MB_ERR_ARG, "null ode");
    if (o->dev.precision != MB_PREC_FP64) return set_err(MB_ERR_ARG, "the device state is pitched FP64 rows only");
    if (sv) *sv = o->dev.sv64;
    if (pitch) *pitch = (size_t)o->dev.ld * sizeof(double);
    return MB_OK;
}

int mb_ode_set_steps(mb_ode *o, double dt, uint32_t num_steps) {
    if (!o || !(dt > 0.0) || num_steps == 0) return set_err(MB_ERR_ARG, "bad arguments");
    o->dev.dt = dt;
    o->dev.num_steps = (int)num_steps;
    return MB_OK;
}

int mb_ode_set_v(mb_ode *o, const double *v, size_t stride) {
    if (!o || !v || stride == 0) return set_err(MB_ERR_ARG, "bad arguments");
    const size_t n = o->dev.n;
    if (stride == 1) {
        /* contiguous: straight from the caller's buffer */
        cudaError_t e = cudaMemcpyAsync(o->dev.sv64, v, n * sizeof(double), cudaMemcpyHostToDevice, o->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(o->stream);
        return e == cudaSuccess ? MB_OK : set_err(MB_ERR_CUDA, "mb_ode_set_v: %s", cudaGetErrorString(e));
    }
    double *tmp = (double *)malloc(n * sizeof(double));
    if (!tmp) return set_err(MB_ERR_NOMEM, "out of host memory");
    for (size_t i = 0; i < n; ++i) tmp[i] = v[i * stride];
    cudaError_t e = cudaMemcpyAsync(o->dev.sv64, tmp, n * sizeof(double), cudaMemcpyHostToDevice, o->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(o->stream);
    free(tmp);
    return e == cudaSuccess ? MB_OK : set_err(MB_ERR_CUDA, "mb_ode_set_v: %s", cudaGetErrorString(e));
}

int mb_ode_get_v(mb_ode *o, double *v, size_t stride) {
    if (!o || !v || stride == 0) return set_err(MB_ERR_ARG, "bad arguments");
    const size_t n = o->dev.n;
    if (stride == 1) {
        cudaError_t e = cudaMemcpyAsync(v, o->dev.sv64, n * sizeof(double), cudaMemcpyDeviceToHost, o->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(o->stream);
        return e == cudaSuccess ? MB_OK : set_err(MB_ERR_CUDA, "mb_ode_get_v: %s", cudaGetErrorString(e));
    }
    double *tmp = (double *)malloc(n * sizeof(double));
    if (!tmp) return set_err(MB_ERR_NOMEM, "out of host memory");
    cudaError_t e = cudaMemcpyAsync(tmp, o->dev.sv64, n * sizeof(double), cudaMemcpyDeviceToHost, o->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(o->stream);
    if (e == cudaSuccess)
        for (size_t i = 0; i < n; ++i) v[i * stride] = tmp[i];
    free(tmp);
    return e == cudaSuccess ? MB_OK : set_err(MB_ERR_CUDA, "mb_ode_get_v: %s", cudaGetErrorString(e));
}

/* ---- monodomain tissue --------------------------------------------------- */

/* struct mb_monodomain: mb_tissue.h */

void mb_monodomain_desc_defaults(mb_monodomain_desc *d) {
    memset(d, 0, sizeof *d);
    d->dx = d->dy = d->dz = 100.0;
    d->dt_pde = 0.02;
    d->dt_ode = 0.02;
    d->beta = 0.14;
    d->cm = 1.0;
    d->model = MB_MODEL_TT2006;
    d->precision = MB_PREC_FP64;
    d->rl_rule = MB_RL_REFERENCE_CPU;
    d->assembly = MB_ASSEMBLY_HOMOGENEOUS;
    d->sigma[0] = d->sigma[1] = d->sigma[2] = 0.00013;
    d->cg_tolerance = 1e-16;
    d->cg_max_iterations = 200;
    d->use_preconditioner = 1;
    d->initial_v = NAN;
    d->track_activation = 0;
    d->activation_threshold = -30.0;
    d->activation_min_interval = 10.0;
    d->ode_adaptive = MB_ODE_FIXED;
    d->ode_abs_tol = 1e-5;
    d->ode_rel_tol = 1e-5;
}

/* alpha = ((beta * cm) / dt) * UM2_TO_CM2 * (dx dy dz), with UM2_TO_CM2 the
 * float literal 1e-8f (monodomain/constants.h:10-11). */
double mb_alpha(double beta, double cm, double dt, double dx, double dy, double dz) {
    return (((beta * cm) / dt) * (double)0.00000001f) * ((dx * dy) * dz);
}

static void destroy_graphs(mb_monodomain *m) {
    if (m->ge_step) cudaGraphExecDestroy(m->ge_step);
    if (m->g_step) cudaGraphDestroy(m->g_step);
    if (m->ge_cg) cudaGraphExecDestroy(m->ge_cg);
    if (m->g_cg) cudaGraphDestroy(m->g_cg);
    m->ge_step = NULL; m->g_step = NULL; m->ge_cg = NULL; m->g_cg = NULL;
}

void mb_monodomain_destroy(mb_monodomain *m) {
    if (!m) return;
    if (m->stream) cudaStreamSynchronize(m->stream);
    destroy_graphs(m);
    void *bufs[] = {m->d_pb, m->d_ppart, m->d_pb32, m->d_bar, m->d_status, m->d_invd, m->d_invd32, m->d_z, m->d_z32,
                    m->d_rtrue, m->d_ap, m->d_ap32, m->d_ap32b, m->d_ecg_leads, m->d_ecg_part, m->d_ecg_log,
                    m->d_mask, m->d_cells, m->d_v, m->d_vstar, m->d_r, m->d_p, m->d_r32, m->d_p32,
                    m->d_partials, m->d_sv64, m->d_sv32, m->d_stim_bits, m->d_celltype, m->d_scale,
                    m->d_fx, m->d_fy, m->d_fz, m->d_table, m->d_table32, m->d_code, m->d_rowid, m->d_act,
                    m->d_stim_host, m->d_ctrl, m->d_log, m->d_stim2[0], m->d_stim2[1], m->d_vsnap[0],
                    m->d_vsnap[1], m->pcg.zc_inv64, m->pcg.zc_inv32, m->pcg.zc_ptab32, m->pcg.zc_maps, m->pcg.zc_w};
    for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; ++i) cudaFree(bufs[i]);
    for (int i = 0; i < 4; ++i) if (m->ev[i]) cudaEventDestroy(m->ev[i]);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 2; ++j) if (m->hev[i][j]) cudaEventDestroy(m->hev[i][j]);
    if (m->copy_stream) cudaStreamDestroy(m->copy_stream);
    if (m->h2d_stream) cudaStreamDestroy(m->h2d_stream);
    if (m->stream) cudaStreamDestroy(m->stream);
    free(m->h_mask);
    free(m);
}

/* Does stim config s cover the cell with centre c?  Same comparisons as the
 * reference stimulus functions. */
static int stim_covers(const mb_stim *s, const double c[3], int64_t g) {
    switch (s->kind) {
    case MB_STIM_X_LESS_THAN: return c[0] < s->x_limit;                       /* stimuli.c:82 */
    case MB_STIM_X_Y_LIMITS:                                                    /* stimuli.c:455-456 */
        return (c[0] >= s->min[0]) && (c[0] <= s->max[0]) && (c[1] >= s->min[1]) && (c[1] <= s->max[1]);
    case MB_STIM_X_Y_Z_LIMITS:                                                  /* stimuli.c:505-507 */
        return (c[0] >= s->min[0]) && (c[0] <= s->max[0]) && (c[1] >= s->min[1]) && (c[1] <= s->max[1]) &&
               (c[2] >= s->min[2]) && (c[2] <= s->max[2]);
    case MB_STIM_CELL_MASK: return s->cell_mask ? s->cell_mask[g] != 0 : 0;
    default: return 0;
    }
}

#define ALLOC(ptr, bytes)                                                                  \
    do {                                                                                   \
        cudaError_t e_ = cudaMalloc((void **)&(ptr), (bytes));                             \
        if (e_ != cudaSuccess) {                                                           \
            rc = set_err(MB_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", (size_t)(bytes),      \
                         cudaGetErrorString(e_));                                          \
            goto fail;                                                                     \
        }                                                                                  \
    } while (0)

#define UPLOAD(dst, src, bytes)                                                            \
    do {                                                                                   \
        cudaError_t e_ = cudaMemcpy((dst), (src), (bytes), cudaMemcpyHostToDevice);        \
        if (e_ != cudaSuccess) {                                                           \
            rc = set_err(MB_ERR_CUDA, "cudaMemcpy failed: %s", cudaGetErrorString(e_));    \
            goto fail;                                                                     \
        }                                                                                  \
    } while (0)

/* The mixed CG's FP32 recurrence runs down to MB_REFINE_MARGIN x tol before
 * the FP64 true residual is evaluated (the stopping test itself is on the
 * FP64 residual against tol).  MB_REFINE_MARGIN in the environment
 * overrides it (tuning). */
#define MB_REFINE_MARGIN 1.0

static int build_graphs(mb_monodomain *m);
static int ode_autotune(mb_monodomain *m);

/* V was written from outside the solve: the fused CG's stored A x no longer
 * belongs to it (stream-ordered) */
static void forget_stored_product(mb_monodomain *m) {
    if (m->d_ctrl) cudaMemsetAsync(&m->d_ctrl->w_valid, 0, sizeof(int32_t), m->stream);
}

/* The start of a loop step: the ECG record of V_n when one is due
 * (monodomain_solver.c:654-657), then the cell models. */
static int step_ode(mb_monodomain *m) {
    if (m->use_ecg) {
        const int e = mbk_ecg(&m->st, m->d_v, &m->ecg, m->d_ctrl, m->stream);
        if (e) return e;
    }
    return mbk_ode_step(&m->ode, m->d_ctrl, m->d_v, m->d_vstar, m->stream);
}

static int pcg_launch(const mb_pcg_dev *q, cudaStream_t s) {
    switch (q->form) {
    case MB_PCG_TILED: return mbk_tcg_launch(q, s);
    case MB_PCG_RESIDENT: return mbk_rcg_launch(q, s);
    case MB_PCG_ZMARCH: return mbk_zcg_launch(q, s);
    default: return mbk_fcg_launch(q, s);
    }
}

/* Picks the CG kernel: every launch-shape variant of the flat persistent
 * kernel, the 2.5D tiled one, where its tiles fit the resident one and, for
 * the 27-point class-table operator, every variant of the z-march kernel
 * solve the tissue's first system (b = alpha V* from the initial state)
 * twice; V is restored after every trial and the fastest by CUDA events is
 * kept.  MB_CG_VARIANT=<n> forces a choice (n = number of flat variants
 * selects the tiled kernel, n + 1 the resident kernel, n + 2 + v z-march
 * variant v). */
static int cg_autotune(mb_monodomain *m) {
    if (!m->use_pcg) return MB_OK;
    const int mixed = m->pcg.mixed;
    const int kind = m->st.kind;
    const int nv = mbk_fcg_variants(kind);
    int resident = mbk_rcg_plan(&m->pcg);
    if (resident && !m->d_rtrue) {
        if (cudaMalloc((void **)&m->d_rtrue, (size_t)m->n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            m->d_rtrue = NULL;
            resident = 0;
        }
        m->pcg.rtrue = m->d_rtrue;
    }
    const int zmarch = mbk_zcg_usable(&m->st) && m->pcg.zc_maps != NULL;
    const int nzv = mbk_zcg_variants();
    const char *env = getenv("MB_CG_VARIANT");
    /* candidates 0..nv-1 flat, nv tiled, nv+1 resident, nv+2.. z-march */
    int lo = 0, hi = nv + 1 + (zmarch ? nzv : 0);
    if (env) lo = hi = atoi(env);
    double *vsave = NULL;
    if (cudaMalloc((void **)&vsave, (size_t)m->n * sizeof(double)) != cudaSuccess)
        return set_err(MB_ERR_NOMEM, "CG tuning buffer");
    cudaMemcpyAsync(vsave, m->d_v, (size_t)m->n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
    float best = 1e30f;
    int bestc = 0, rc = MB_OK;      /* variant 0 runs on every grid */
    for (int cand = lo; cand <= hi && !rc; ++cand) {
        mb_pcg_dev q = m->pcg;
        if (cand < nv) {
            q.form = MB_PCG_FLAT;
            q.variant = cand;
            q.blocks = mbk_fcg_max_blocks(mixed, kind, cand);
        } else if (cand == nv) {
            q.form = MB_PCG_TILED;
            const int items = q.tiles_x * q.tiles_y * q.nchunks;
            const int mb = mbk_tcg_max_blocks(mixed);
            q.blocks = items < mb ? items : mb;
        } else if (cand == nv + 1) {
            if (!resident) continue;
            q.form = MB_PCG_RESIDENT;
            q.blocks = q.rc_nbx * q.rc_nby;
        } else {
            if (!zmarch || cand - nv - 2 >= nzv) continue;
            q.form = MB_PCG_ZMARCH;
            q.zc_variant = cand - nv - 2;
            q.blocks = mbk_zcg_max_blocks(mixed, q.zc_variant);
        }
        if (q.blocks <= 0) continue;
        if (cand < nv && mbk_fcg_variant_groups(cand) && (m->desc.nx % 4) != 0) continue;
        float tsum = 0;
        for (int rep = 0; rep < 3 && !rc; ++rep) {
            cudaMemcpyAsync(m->d_v, vsave, (size_t)m->n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
            forget_stored_product(m);
            cudaEventRecord(m->ev[0], m->stream);
            const int e = pcg_launch(&q, m->stream);
            cudaEventRecord(m->ev[1], m->stream);
            if (e || cudaEventSynchronize(m->ev[1]) != cudaSuccess) {
                rc = set_err(MB_ERR_CUDA, "CG tuning launch failed (candidate %d): %s", cand,
                             cudaGetErrorString(e ? (cudaError_t)e : cudaGetLastError()));
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]);
            if (rep > 0) tsum += ms;      /* first run warms up */
        }
        if (!rc && tsum < best) {
            best = tsum;
            bestc = cand;
        }
    }
    cudaMemcpyAsync(m->d_v, vsave, (size_t)m->n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
    forget_stored_product(m);
    cudaStreamSynchronize(m->stream);
    cudaFree(vsave);
    if (rc) return rc;
    int st = 0;
    cudaMemcpy(&st, m->d_status, sizeof st, cudaMemcpyDeviceToHost);
    if (st) return set_err(MB_ERR_CUDA, "CG grid barrier timed out during tuning");
    if (bestc < nv) {
        m->pcg.form = MB_PCG_FLAT;
        m->pcg.variant = bestc;
        m->pcg.blocks = mbk_fcg_max_blocks(mixed, kind, bestc);
    } else if (bestc == nv) {
        m->pcg.form = MB_PCG_TILED;
        const int items = m->pcg.tiles_x * m->pcg.tiles_y * m->pcg.nchunks;
        const int mb = mbk_tcg_max_blocks(mixed);
        m->pcg.blocks = items < mb ? items : mb;
    } else if (bestc == nv + 1) {
        m->pcg.form = MB_PCG_RESIDENT;
        m->pcg.blocks = m->pcg.rc_nbx * m->pcg.rc_nby;
    } else {
        m->pcg.form = MB_PCG_ZMARCH;
        m->pcg.zc_variant = bestc - nv - 2;
        m->pcg.blocks = mbk_zcg_max_blocks(mixed, m->pcg.zc_variant);
    }
    if (m->pcg.form != MB_PCG_RESIDENT && m->d_rtrue) {
        cudaFree(m->d_rtrue);
        m->d_rtrue = NULL;
        m->pcg.rtrue = NULL;
    }
    m->cg_tune_ms = best / 2.0f;
    return MB_OK;
}

int mb_monodomain_create(mb_monodomain **out, const mb_monodomain_desc *d) {
    int rc = MB_OK;
    uint32_t *cells = NULL;
    uint8_t *bits = NULL, *ct = NULL;
    float *scale = NULL;
    double *vinit = NULL;
    mb_assembly_out asmb;
    memset(&asmb, 0, sizeof asmb);
    if (!out || !d) return set_err(MB_ERR_ARG, "null argument");
    *out = NULL;
    if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0) return set_err(MB_ERR_ARG, "grid dimensions must be positive");
    if (!(d->dx > 0 && d->dy > 0 && d->dz > 0 && d->dt_pde > 0 && d->dt_ode > 0))
        return set_err(MB_ERR_ARG, "dx, dy, dz, dt_pde and dt_ode must be positive");
    if (d->num_stims < 0 || d->num_stims > MB_MAX_STIMS) return set_err(MB_ERR_ARG, "num_stims out of range");
    if (d->precision != MB_PREC_FP64 && d->precision != MB_PREC_MIXED) return set_err(MB_ERR_ARG, "bad precision");
    if (d->ode_adaptive) {
        if (d->model != MB_MODEL_TORORD_FKATP_ENDO)
            return set_err(MB_ERR_ARG, "the adaptive ODE step belongs to the forward-Euler library (ToRORd_fkatp_endo)");
        if (d->ode_adaptive != MB_ODE_ADAPTIVE_CPU && d->ode_adaptive != MB_ODE_ADAPTIVE_GPU)
            return set_err(MB_ERR_ARG, "bad ode_adaptive");
        if (!(d->ode_abs_tol > 0 && d->ode_rel_tol > 0 && d->dt_ode <= d->dt_pde))
            return set_err(MB_ERR_ARG, "adaptive ODE step: tolerances must be positive and dt_ode <= dt_pde");
    }
    if (d->model == MB_MODEL_TORORD_FKATP_ENDO && (d->celltype || d->current_scale))
        return set_err(MB_ERR_ARG, "ToRORd_fkatp_endo takes no cell types or conductance scalings");
    int neq;
    double model_v0;
    if (mb_init_cell_model_data(d->model, &neq, &model_v0)) return MB_ERR_ARG;
    const int64_t n = (int64_t)d->nx * d->ny * d->nz;
    if (n > 0x7fffffffLL) return set_err(MB_ERR_ARG, "grid too large (%lld cells)", (long long)n);

    mb_monodomain *m = (mb_monodomain *)calloc(1, sizeof *m);
    if (!m) return set_err(MB_ERR_NOMEM, "out of host memory");
    m->desc = *d;
    m->neq = neq;
    m->n = n;
    m->use_graphs = getenv("MB_NO_GRAPH") == NULL;
    /* num_steps = (int)(dt_pde / dt_ode) (monodomain_solver.c:510-520) */
    m->num_steps = d->dt_pde >= d->dt_ode ? (int)(d->dt_pde / d->dt_ode) : 1;
    if (m->num_steps < 1) m->num_steps = 1;

    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        rc = set_err(MB_ERR_CUDA, "cudaStreamCreate failed");
        goto fail;
    }
    for (int i = 0; i < 4; ++i) cudaEventCreate(&m->ev[i]);

    /* active cells, compact numbering in grid order */
    uint32_t na = 0;
    if (d->active) {
        cells = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
        if (!cells) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (int64_t g = 0; g < n; ++g) if (d->active[g]) cells[na++] = (uint32_t)g;
    } else {
        na = (uint32_t)n;
    }
    m->n_active = na;
    if (na == 0) { rc = set_err(MB_ERR_ARG, "no active cells"); goto fail; }
    const uint32_t ld = round_up32(na);

    /* ODE state */
    int n64, n32;
    ode_rows(d->model, d->precision, d->ode_adaptive, &n64, &n32);
    ALLOC(m->d_sv64, (size_t)n64 * ld * sizeof(double));
    if (n32) ALLOC(m->d_sv32, (size_t)n32 * ld * sizeof(float));
    m->ode.model = d->model;
    m->ode.precision = d->model == MB_MODEL_TORORD_FKATP_ENDO ? MB_PREC_FP64 : d->precision;
    m->ode.rl_rule = d->rl_rule;
    if (d->ode_adaptive) {
        /* one adaptive pass per loop step (monodomain_solver.c:517-527) */
        m->num_steps = 1;
        m->ode.adaptive = d->ode_adaptive;
        m->ode.min_dt = d->dt_ode > 0.0 ? d->dt_ode : 1e-10;
        m->ode.max_dt = d->dt_pde;
        m->ode.abs_tol = d->ode_abs_tol;
        m->ode.rel_tol = d->ode_rel_tol;
        m->ode.adapt_span = d->ode_adaptive == MB_ODE_ADAPTIVE_CPU ? m->ode.min_dt : m->ode.max_dt;
    }
    m->ode.num_steps = m->num_steps;
    m->ode.n = na;
    m->ode.ld = ld;
    m->ode.sv64 = m->d_sv64;
    m->ode.sv32 = m->d_sv32;
    m->ode.dt = d->dt_ode;
    if (d->active) {
        ALLOC(m->d_mask, (size_t)n);
        UPLOAD(m->d_mask, d->active, (size_t)n);
        ALLOC(m->d_cells, (size_t)na * sizeof(uint32_t));
        UPLOAD(m->d_cells, cells, (size_t)na * sizeof(uint32_t));
        m->ode.cell = m->d_cells;
    }

    /* stimulus bits per compact cell */
    if (d->num_stims > 0) {
        bits = (uint8_t *)calloc(na, 1);
        if (!bits) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        int any = 0;
        for (uint32_t t = 0; t < na; ++t) {
            const int64_t g = cells ? cells[t] : t;
            const int i = (int)(g % d->nx), j = (int)((g / d->nx) % d->ny), k = (int)(g / ((int64_t)d->nx * d->ny));
            const double c[3] = {(i + 0.5) * d->dx, (j + 0.5) * d->dy, (k + 0.5) * d->dz};
            for (int s = 0; s < d->num_stims; ++s)
                if (stim_covers(&d->stims[s], c, g)) { bits[t] |= (uint8_t)(1u << s); any = 1; }
        }
        if (any) {
            ALLOC(m->d_stim_bits, na);
            UPLOAD(m->d_stim_bits, bits, na);
            m->ode.stim_bits = m->d_stim_bits;
        }
    }
    ALLOC(m->d_stim_host, (size_t)na * sizeof(double));

    /* cell types (ToRORd transmurality) and conductance scalings, compacted */
    if (d->celltype && d->model == MB_MODEL_TORORD_FKATP_MIXED) {
        ct = (uint8_t *)malloc(na);
        if (!ct) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (uint32_t t = 0; t < na; ++t) ct[t] = d->celltype[cells ? cells[t] : t];
        ALLOC(m->d_celltype, na);
        UPLOAD(m->d_celltype, ct, na);
        m->ode.celltype = m->d_celltype;
    }
    if (d->current_scale) {
        scale = (float *)calloc((size_t)MB_NUM_SCALES * ld, sizeof(float));
        if (!scale) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (int q = 0; q < MB_NUM_SCALES; ++q)
            for (uint32_t t = 0; t < na; ++t) scale[(size_t)q * ld + t] = (float)d->current_scale[(size_t)q * n + (cells ? cells[t] : t)];
        ALLOC(m->d_scale, (size_t)MB_NUM_SCALES * ld * sizeof(float));
        UPLOAD(m->d_scale, scale, (size_t)MB_NUM_SCALES * ld * sizeof(float));
        m->ode.scale = m->d_scale;
    }

    /* initial conditions of the ODE state */
    {
        double table[3 * MB_MAX_NEQ];
        int ntypes;
        model_ic_table(d->model, d->initial_state, table, &ntypes);
        double *d_table = NULL;
        ALLOC(d_table, sizeof table);
        UPLOAD(d_table, table, sizeof table);
        int e = mbk_ode_init(&m->ode, d_table, ntypes, m->stream);
        cudaStreamSynchronize(m->stream);
        cudaFree(d_table);
        if (e) { rc = set_err(MB_ERR_CUDA, "ode init: %s", cudaGetErrorString((cudaError_t)e)); goto fail; }
    }
    if (m->ode.adaptive) {
        /* per-cell dt = min_dt, time_new = previous_dt = 0
         * (ToRORd_fkatp_endo.c:14-25) */
        double *rows = (double *)calloc((size_t)3 * ld, sizeof(double));
        if (!rows) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (uint32_t t = 0; t < ld; ++t) rows[t] = m->ode.min_dt;
        cudaError_t e = cudaMemcpy(m->d_sv64 + (size_t)neq * ld, rows, (size_t)3 * ld * sizeof(double),
                                   cudaMemcpyHostToDevice);
        free(rows);
        if (e != cudaSuccess) { rc = set_err(MB_ERR_CUDA, "adaptive rows: %s", cudaGetErrorString(e)); goto fail; }
    }

    /* V (grid): the CG initial guess is the assembly init value
     * (set_initial_conditions_fvm); V* starts at the ODE state's own V so that
     * the first ODE step reads sv[0] (update_ode_state_vector is skipped at t = 0). */
    ALLOC(m->d_v, (size_t)n * sizeof(double));
    ALLOC(m->d_vstar, (size_t)n * sizeof(double));
    {
        const double v0 = isnan(d->initial_v) ? model_v0 : d->initial_v;
        vinit = (double *)malloc((size_t)n * sizeof(double));
        if (!vinit) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (int64_t g = 0; g < n; ++g) vinit[g] = (!d->active || d->active[g]) ? v0 : 0.0;
        UPLOAD(m->d_v, vinit, (size_t)n * sizeof(double));
        CKK(cudaMemset(m->d_vstar, 0, (size_t)n * sizeof(double)));
        /* V* <- state V (row 0 of the ODE table rows) */
        double *dense = NULL;
        ALLOC(dense, (size_t)neq * na * sizeof(double));
        mbk_ode_gather(&m->ode, NULL, dense, m->stream);
        mb_ode_dev tmp = m->ode;
        int e = mbk_ode_scatter(&tmp, dense, m->d_vstar, m->stream);
        cudaStreamSynchronize(m->stream);
        cudaFree(dense);
        if (e) { rc = set_err(MB_ERR_CUDA, "V* init failed"); goto fail; }
    }

    rc = ode_autotune(m);
    if (rc) goto fail;

    /* diffusion operator */
    m->st.nx = d->nx; m->st.ny = d->ny; m->st.nz = d->nz;
    m->st.alpha = mb_alpha(d->beta, d->cm, d->dt_pde, d->dx, d->dy, d->dz);
    m->st.mask = m->d_mask;
    rc = mb_assemble(d, &asmb);
    if (rc) goto fail;
    m->st.kind = asmb.kind;
    m->st.cx = asmb.cx; m->st.cy = asmb.cy; m->st.cz = asmb.cz;
    if (asmb.kind == 1) {
        ALLOC(m->d_fx, (size_t)n * sizeof(double));
        ALLOC(m->d_fy, (size_t)n * sizeof(double));
        ALLOC(m->d_fz, (size_t)n * sizeof(double));
        UPLOAD(m->d_fx, asmb.fx, (size_t)n * sizeof(double));
        UPLOAD(m->d_fy, asmb.fy, (size_t)n * sizeof(double));
        UPLOAD(m->d_fz, asmb.fz, (size_t)n * sizeof(double));
        m->st.fx = m->d_fx; m->st.fy = m->d_fy; m->st.fz = m->d_fz;
    } else if (asmb.kind == 2) {
        const size_t tn = (size_t)d->nz * 9 * 27;
        ALLOC(m->d_table, tn * sizeof(double));
        UPLOAD(m->d_table, asmb.table, tn * sizeof(double));
        float *t32 = (float *)malloc(tn * sizeof(float));
        if (!t32) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (size_t q = 0; q < tn; ++q) t32[q] = (float)asmb.table[q];
        ALLOC(m->d_table32, tn * sizeof(float));
        cudaMemcpy(m->d_table32, t32, tn * sizeof(float), cudaMemcpyHostToDevice);
        free(t32);
        m->st.table = m->d_table; m->st.table32 = m->d_table32;
        uint32_t nzm = 1u << 13;
        for (size_t q = 0; q < tn; ++q)
            if (asmb.table[q] != 0.0) nzm |= 1u << (q % 27);
        m->st.nzmask = nzm;
    }
    /* per-cell row codes read by the persistent CG */
    if (m->st.kind == 2) {
        if ((int64_t)d->nz * 9 > 65535) { rc = set_err(MB_ERR_UNSUPPORTED, "nz above 7281 for a per-plane operator"); goto fail; }
        ALLOC(m->d_rowid, (size_t)n * sizeof(uint16_t));
    } else {
        ALLOC(m->d_code, (size_t)n);
    }
    m->st.code = m->d_code;
    m->st.rowid = m->d_rowid;
    CKK(mbk_stencil_codes(&m->st, m->d_code, m->d_rowid, m->stream));

    /* CG work vectors */
    m->cg.precision = d->precision;
    {
        int gb = (int)((n + 255) / 256);
        if (gb > mbk_max_grid_blocks()) gb = mbk_max_grid_blocks();
        if (gb < 1) gb = 1;
        m->cg.grid_blocks = gb;
        ALLOC(m->d_partials, (size_t)3 * gb * sizeof(double));
    }
    if (d->precision == MB_PREC_FP64) {
        ALLOC(m->d_r, (size_t)n * sizeof(double));
        ALLOC(m->d_p, (size_t)n * sizeof(double));
        CKK(cudaMemset(m->d_r, 0, (size_t)n * sizeof(double)));
        CKK(cudaMemset(m->d_p, 0, (size_t)n * sizeof(double)));
    } else {
        ALLOC(m->d_r32, (size_t)n * sizeof(float));
        ALLOC(m->d_p32, (size_t)n * sizeof(float));
        CKK(cudaMemset(m->d_r32, 0, (size_t)n * sizeof(float)));
        CKK(cudaMemset(m->d_p32, 0, (size_t)n * sizeof(float)));
    }
    m->cg.x = m->d_v;
    m->cg.vstar = m->d_vstar;
    m->cg.r = m->d_r; m->cg.p = m->d_p;
    m->cg.r32 = m->d_r32; m->cg.p32 = m->d_p32;
    m->cg.partials = m->d_partials;

    /* persistent cooperative CG: one launch per solve */
    {
        const char *mode = getenv("MB_CG");
        m->use_pcg = !(mode && strcmp(mode, "graph") == 0);
        const int mixed = d->precision == MB_PREC_MIXED;
        int maxb = -1;
        if (m->use_pcg) {
            /* the partials buffer must fit the largest grid of any variant */
            const int nv = mbk_fcg_variants(m->st.kind);
            for (int v = 0; v < nv; ++v) {
                const int b = mbk_fcg_max_blocks(mixed, m->st.kind, v);
                if (b > maxb) maxb = b;
            }
            const int bt = mbk_tcg_max_blocks(mixed);
            if (bt > maxb) maxb = bt;
            if (mbk_zcg_usable(&m->st))
                for (int v = 0; v < mbk_zcg_variants(); ++v) {
                    const int b = mbk_zcg_max_blocks(mixed, v);
                    if (b > maxb) maxb = b;
                }
            mbk_tcg_layout(d->nx, d->ny, d->nz, bt > 0 ? bt : 1, &m->pcg.tiles_x, &m->pcg.tiles_y, &m->pcg.zchunk,
                           &m->pcg.nchunks);
        }
        if (maxb <= 0) m->use_pcg = 0;
        if (m->use_pcg) {
            const int blocks = maxb;
            if (d->precision == MB_PREC_FP64) {
                ALLOC(m->d_pb, (size_t)n * sizeof(double));
                CKK(cudaMemset(m->d_pb, 0, (size_t)n * sizeof(double)));
                ALLOC(m->d_z, (size_t)n * sizeof(double));
                CKK(cudaMemset(m->d_z, 0, (size_t)n * sizeof(double)));
                ALLOC(m->d_ap, (size_t)n * sizeof(double));
                CKK(cudaMemset(m->d_ap, 0, (size_t)n * sizeof(double)));
            } else {
                ALLOC(m->d_pb32, (size_t)n * sizeof(float));
                CKK(cudaMemset(m->d_pb32, 0, (size_t)n * sizeof(float)));
                ALLOC(m->d_z32, (size_t)n * sizeof(float));
                CKK(cudaMemset(m->d_z32, 0, (size_t)n * sizeof(float)));
                ALLOC(m->d_ap32, (size_t)n * sizeof(float));
                CKK(cudaMemset(m->d_ap32, 0, (size_t)n * sizeof(float)));
                if (mbk_zcg_usable(&m->st)) {
                    /* the z-march fused pass alternates A p between two buffers */
                    ALLOC(m->d_ap32b, (size_t)n * sizeof(float));
                    CKK(cudaMemset(m->d_ap32b, 0, (size_t)n * sizeof(float)));
                }
            }
            ALLOC(m->d_ppart, ((size_t)16 * blocks + 16) * sizeof(double));
            if (d->precision == MB_PREC_FP64) {
                ALLOC(m->d_invd, (size_t)n * sizeof(double));
                CKK(cudaMemset(m->d_invd, 0, (size_t)n * sizeof(double)));
            } else {
                ALLOC(m->d_invd32, (size_t)n * sizeof(float));
                CKK(cudaMemset(m->d_invd32, 0, (size_t)n * sizeof(float)));
            }
            CKK(mbk_inv_diag(&m->st, m->d_invd, m->d_invd32, m->stream));
            if (mbk_zcg_usable(&m->st)) {
                ALLOC(m->pcg.zc_inv64, (size_t)d->nz * 9 * sizeof(double));
                ALLOC(m->pcg.zc_inv32, (size_t)d->nz * 9 * sizeof(float));
                ALLOC(m->pcg.zc_ptab32, (size_t)d->nz * mbk_zcg_ptab_floats() * sizeof(float));
                /* the fused mixed solve's stored A x (its next solve's starting product) */
                if (d->precision == MB_PREC_MIXED) ALLOC(m->pcg.zc_w, (size_t)n * sizeof(double));
                CKK(mbk_zcg_inv_tables(&m->st, m->pcg.zc_inv64, m->pcg.zc_inv32, m->pcg.zc_ptab32, m->stream));
            }
            CKK(cudaStreamSynchronize(m->stream));
            ALLOC(m->d_bar, 2 * sizeof(unsigned));
            ALLOC(m->d_status, sizeof(int));
            CKK(cudaMemset(m->d_bar, 0, 2 * sizeof(unsigned)));
            CKK(cudaMemset(m->d_status, 0, sizeof(int)));
            mb_pcg_dev *q = &m->pcg;
            q->mixed = d->precision == MB_PREC_MIXED;
            q->form = MB_PCG_FLAT;
            q->variant = 0;
            q->rc_shape = -1;
            q->rtrue = NULL;
            q->blocks = mbk_fcg_max_blocks(mixed, m->st.kind, 0);
            q->x = m->d_v;
            q->vstar = m->d_vstar;
            q->b = NULL;
            q->r64 = m->d_r; q->pa64 = m->d_p; q->pb64 = m->d_pb;
            q->r32 = m->d_r32; q->pa32 = m->d_p32; q->pb32 = m->d_pb32;
            q->z64 = m->d_z; q->z32 = m->d_z32;
            q->ap64 = m->d_ap; q->ap32 = m->d_ap32; q->ap32b = m->d_ap32b;
            q->partials = m->d_ppart;
            q->inv_diag64 = m->d_invd;
            q->inv_diag32 = m->d_invd32;
            q->bar = m->d_bar;
            q->status = m->d_status;
            q->st = m->st;
            if (q->zc_inv64) CKK(mbk_zcg_prepare(q));
        }
    }

    /* pseudo-bidomain ECG records (ecg.cu), taken at step starts */
    if (d->ecg_rate > 0) {
        const int nl = d->ecg_n_leads;
        if (nl < 1 || nl > MB_ECG_MAX_LEADS || !d->ecg_leads || d->ecg_capacity < 1 || !(d->ecg_sigma_b != 0.0)) {
            rc = set_err(MB_ERR_ARG, "ECG: 1..%d leads, a record capacity and a nonzero sigma_b are needed",
                         MB_ECG_MAX_LEADS);
            goto fail;
        }
        ALLOC(m->d_ecg_leads, (size_t)3 * nl * sizeof(double));
        UPLOAD(m->d_ecg_leads, d->ecg_leads, (size_t)3 * nl * sizeof(double));
        ALLOC(m->d_ecg_part, (size_t)MB_ECG_BLOCKS * MB_ECG_MAX_LEADS * sizeof(double));
        ALLOC(m->d_ecg_log, (size_t)d->ecg_capacity * (1 + nl) * sizeof(double));
        mb_ecg_dev *e = &m->ecg;
        e->rate = d->ecg_rate;
        e->n_leads = nl;
        e->capacity = d->ecg_capacity;
        e->dx = d->dx; e->dy = d->dy; e->dz = d->dz;
        e->scale = 1.0 / (4.0 * M_PI * d->ecg_sigma_b);   /* ecg.c:236 */
        e->leads = m->d_ecg_leads;
        e->partials = m->d_ecg_part;
        e->log = m->d_ecg_log;
        m->use_ecg = 1;
    }

    /* activation tracking rows (read and written by the ODE kernels) */
    if (d->track_activation) {
        const size_t ld = m->ode.ld, bytes = (size_t)MB_ACT_ROWS * ld * sizeof(float);
        float *h = (float *)malloc(bytes);
        if (!h) { rc = set_err(MB_ERR_NOMEM, "host memory"); goto fail; }
        for (size_t q = 0; q < ld; ++q) {
            h[MB_ACT_VPREV * ld + q] = NAN;
            h[MB_ACT_FIRST * ld + q] = -1.0f;
            h[MB_ACT_LAST * ld + q] = -1.0f;
            h[MB_ACT_APD * ld + q] = -1.0f;
            h[MB_ACT_VPEAK * ld + q] = 0.0f;
            h[MB_ACT_VREST * ld + q] = 0.0f;
            h[MB_ACT_STATE * ld + q] = 0.0f;
        }
        cudaError_t e = cudaMalloc((void **)&m->d_act, bytes);
        if (e == cudaSuccess) e = cudaMemcpy(m->d_act, h, bytes, cudaMemcpyHostToDevice);
        free(h);
        if (e != cudaSuccess) { rc = set_err(MB_ERR_NOMEM, "activation rows: %s", cudaGetErrorString(e)); goto fail; }
        m->ode.act = m->d_act;
    }

    /* control block */
    {
        mb_ctrl c;
        memset(&c, 0, sizeof c);
        c.cur_time = 0.0;
        c.count = 0;
        c.num_stims = d->num_stims;
        for (int s = 0; s < d->num_stims; ++s) {
            c.stim_start[s] = d->stims[s].start;
            c.stim_dur[s] = d->stims[s].duration;
            c.stim_period[s] = d->stims[s].period;
            c.stim_current[s] = d->stims[s].current;
        }
        c.tol = d->cg_tolerance;
        c.max_its = d->cg_max_iterations > 0 ? d->cg_max_iterations : 200;
        c.use_precond = d->use_preconditioner ? 1 : 0;
        /* the FP32 recurrence is trusted down to refine_ratio x the last
         * FP64 r.r; MB_REFINE_RATIO overrides it (tuning) */
        c.refine_ratio = 1e-10;
        c.refine_floor = MB_REFINE_MARGIN * c.tol;
        {
            const char *env = getenv("MB_REFINE_RATIO");
            if (env && atof(env) > 0.0) c.refine_ratio = atof(env);
            env = getenv("MB_REFINE_MARGIN");
            if (env && atof(env) > 0.0) c.refine_floor = atof(env) * c.tol;
        }
        c.act_dt = d->dt_pde;
        c.act_threshold = (float)(isnan(d->activation_threshold) ? -30.0 : d->activation_threshold);
        c.act_min_interval = (float)(isnan(d->activation_min_interval) ? 10.0 : d->activation_min_interval);
        ALLOC(m->d_ctrl, sizeof(mb_ctrl));
        UPLOAD(m->d_ctrl, &c, sizeof c);
        m->pcg.ctrl = m->d_ctrl;
        m->pcg.st = m->st;
    }
    m->log_len = 1 << 20;
    ALLOC(m->d_log, (size_t)m->log_len * sizeof(mb_step_stats));

    rc = cg_autotune(m);
    if (rc) goto fail;
    rc = build_graphs(m);
    if (rc) goto fail;

    free(cells); free(bits); free(ct); free(scale); free(vinit);
    mb_assembly_free(&asmb);
    /* keep no caller pointers beyond this call */
    if (d->active) {
        m->h_mask = (uint8_t *)malloc((size_t)n);
        if (!m->h_mask) { mb_monodomain_destroy(m); return set_err(MB_ERR_NOMEM, "host memory"); }
        memcpy(m->h_mask, d->active, (size_t)n);
    }
    m->desc.active = m->h_mask;
    m->desc.initial_state = NULL;
    m->desc.celltype = NULL;
    m->desc.current_scale = NULL;
    m->desc.fibre_angle_z = NULL;
    m->desc.sigma_cell = NULL;
    for (int s = 0; s < MB_MAX_STIMS; ++s) m->desc.stims[s].cell_mask = NULL;
    *out = m;
    return MB_OK;
fail:
    free(cells); free(bits); free(ct); free(scale); free(vinit);
    mb_assembly_free(&asmb);
    mb_monodomain_destroy(m);
    return rc ? rc : MB_ERR_CUDA;
}

/* Picks the register-budget variant of the ODE kernel: each variant advances
 * up to 2^20 cells from the current state into scratch buffers (the live
 * state is not touched) and the fastest by CUDA events wins. */
static int ode_autotune(mb_monodomain *m) {
    const char *env = getenv("MB_ODE_VARIANT");
    if (env) {
        m->ode.variant = atoi(env);
        return MB_OK;
    }
    int n64, n32;
    ode_rows(m->desc.model, m->desc.precision, m->desc.ode_adaptive, &n64, &n32);
    /* every cell where the scratch outputs fit in a quarter of the free
     * device memory (launch shapes rank differently on a few waves of blocks
     * than on the hundreds of waves of a large tissue), else 4 M cells */
    uint32_t nt = m->n_active;
    {
        size_t fr = 0, tot = 0;
        const size_t need = ((size_t)n64 * 8 + (size_t)n32 * 4) * nt + (size_t)m->n * 8;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess || need > fr / 4) {
            cudaGetLastError();
            if (nt > (1u << 22)) nt = 1u << 22;
        }
    }
    double *s64 = NULL, *vs = NULL;
    float *s32 = NULL;
    int rc = MB_OK;
    if (cudaMalloc((void **)&s64, (size_t)n64 * nt * sizeof(double)) != cudaSuccess ||
        (n32 && cudaMalloc((void **)&s32, (size_t)n32 * nt * sizeof(float)) != cudaSuccess) ||
        cudaMalloc((void **)&vs, (size_t)m->n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(s64); cudaFree(s32); cudaFree(vs);
        m->ode.variant = 0;
        return MB_OK;           /* no room to tune: keep the default */
    }
    mb_ode_dev t = m->ode;
    t.n = nt;
    t.stim_bits = NULL;
    t.out64 = s64;
    t.out32 = s32;
    t.out_ld = nt;
    float best = 1e30f;
    int bestv = 0;
    for (int v = 0; v < MB_ODE_VARIANTS && !rc; ++v) {
        t.variant = v;
        const int e = mbk_ode_step(&t, NULL, m->d_vstar, vs, m->stream);
        if (e == (int)cudaErrorInvalidConfiguration && v >= 6) continue;   /* staged form does not fit */
        if (e) { rc = set_err(MB_ERR_CUDA, "ODE tuning launch failed"); break; }
        cudaEventRecord(m->ev[0], m->stream);
        for (int q = 0; q < 3; ++q) mbk_ode_step(&t, NULL, m->d_vstar, vs, m->stream);
        cudaEventRecord(m->ev[1], m->stream);
        if (cudaEventSynchronize(m->ev[1]) != cudaSuccess) { rc = set_err(MB_ERR_CUDA, "ODE tuning failed"); break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, m->ev[0], m->ev[1]);
        if (ms < best) { best = ms; bestv = v; }
    }
    cudaFree(s64); cudaFree(s32); cudaFree(vs);
    m->ode.variant = bestv;
    return rc;
}

int mb_cg_launch_shapes(int *flat_shapes) {
    if (!flat_shapes) return set_err(MB_ERR_ARG, "null");
    *flat_shapes = mbk_fcg_variants(0);
    return MB_OK;
}

int mb_monodomain_tuning(mb_monodomain *m, int *ode_variant, int *cg_blocks, int *cg_kernel) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (ode_variant) *ode_variant = m->ode.variant;
    if (cg_blocks) *cg_blocks = m->use_pcg ? m->pcg.blocks : m->cg.grid_blocks;
    if (cg_kernel)
        *cg_kernel = !m->use_pcg ? -1
                   : m->pcg.form == MB_PCG_TILED ? 100
                   : m->pcg.form == MB_PCG_RESIDENT ? 200
                   : m->pcg.form == MB_PCG_ZMARCH ? 300 + m->pcg.zc_variant : m->pcg.variant;
    return MB_OK;
}

/* Captures the launches of fn into a fresh graph. */
typedef int (*capture_fn)(mb_monodomain *m, int in_body);

static int cap_pre(mb_monodomain *m, int in_body) {
    (void)in_body;
    int e = step_ode(m);
    if (!e) e = mbk_cg_init(&m->st, &m->cg, m->d_ctrl, 0ULL, 0, m->stream);
    return e;
}

static int cap_cginit(mb_monodomain *m, int in_body) {
    (void)in_body;
    return mbk_cg_init(&m->st, &m->cg, m->d_ctrl, 0ULL, 0, m->stream);
}

static int cap_post(mb_monodomain *m, int in_body) {
    (void)in_body;
    return mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream);
}

/* The CG body captured into the conditional node's body graph, given the
 * node's handle (per tissue, passed down: tissues created concurrently from
 * several host threads each capture their own). */
static int cap_body(mb_monodomain *m, unsigned long long cond) {
    return mbk_cg_body(&m->st, &m->cg, m->d_ctrl, cond, 1, m->stream);
}

static int capture_graph(mb_monodomain *m, capture_fn fn, cudaGraph_t *out) {
    CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    int e = fn(m, 0);
    cudaGraph_t g = NULL;
    cudaError_t ee = cudaStreamEndCapture(m->stream, &g);
    if (e) return set_err(MB_ERR_CUDA, "launch during capture failed: %s", cudaGetErrorString((cudaError_t)e));
    if (ee != cudaSuccess) return set_err(MB_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ee));
    *out = g;
    return MB_OK;
}

/* graph = [child pre] -> WHILE(cond){ body } -> [child post]  (post optional) */
static int build_loop_graph(mb_monodomain *m, capture_fn pre, capture_fn post, cudaGraph_t *out,
                            cudaGraphExec_t *exec_out) {
    cudaGraph_t g = NULL, gpre = NULL, gpost = NULL;
    CK(cudaGraphCreate(&g, 0));
    int rc = capture_graph(m, pre, &gpre);
    if (rc) return rc;
    cudaGraphNode_t npre, ncond, npost;
    CK(cudaGraphAddChildGraphNode(&npre, g, NULL, 0, gpre));
    cudaGraphDestroy(gpre);

    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    struct cudaGraphNodeParams cp;
    memset(&cp, 0, sizeof cp);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    CK(cudaGraphAddNode(&ncond, g, &npre, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(m->stream, body, NULL, NULL, 0, cudaStreamCaptureModeThreadLocal));
    int e = cap_body(m, (unsigned long long)h);
    cudaGraph_t body_out = NULL;
    cudaError_t ee = cudaStreamEndCapture(m->stream, &body_out);
    if (e) return set_err(MB_ERR_CUDA, "CG body capture failed: %s", cudaGetErrorString((cudaError_t)e));
    if (ee != cudaSuccess) return set_err(MB_ERR_CUDA, "CG body capture: %s", cudaGetErrorString(ee));

    if (post) {
        rc = capture_graph(m, post, &gpost);
        if (rc) return rc;
        CK(cudaGraphAddChildGraphNode(&npost, g, &ncond, 1, gpost));
        cudaGraphDestroy(gpost);
    }
    CK(cudaGraphInstantiate(exec_out, g, 0));
    *out = g;
    return MB_OK;
}

static int cap_pcg_step(mb_monodomain *m, int in_body) {
    (void)in_body;
    int e = step_ode(m);
    if (!e) e = pcg_launch(&m->pcg, m->stream);
    if (!e) e = mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream);
    return e;
}

static int build_graphs(mb_monodomain *m) {
    if (!m->use_graphs) return MB_OK;
    int rc;
    if (m->use_pcg) {
        rc = capture_graph(m, cap_pcg_step, &m->g_step);
        if (!rc) CK(cudaGraphInstantiate(&m->ge_step, m->g_step, 0));
    } else {
        rc = build_loop_graph(m, cap_pre, cap_post, &m->g_step, &m->ge_step);
        if (!rc) rc = build_loop_graph(m, cap_cginit, NULL, &m->g_cg, &m->ge_cg);
    }
    if (rc) {
        /* fall back to host-driven launches */
        cudaGetLastError();
        destroy_graphs(m);
        m->use_graphs = 0;
        if (getenv("MB_REQUIRE_GRAPH")) return rc;
    }
    return MB_OK;
}

int mb_monodomain_uses_graphs(mb_monodomain *m) { return m ? m->use_graphs : 0; }

/* Host-driven CG loop (no conditional graph): iterations in chunks, the
 * stopping flag read back between chunks. */
static int cg_host_loop(mb_monodomain *m) {
    CKK(mbk_cg_init(&m->st, &m->cg, m->d_ctrl, 0ULL, 0, m->stream));
    const int chunk = 8;
    for (int it = 0; it < m->desc.cg_max_iterations + 2; it += chunk) {
        for (int q = 0; q < chunk; ++q) CKK(mbk_cg_body(&m->st, &m->cg, m->d_ctrl, 0ULL, 0, m->stream));
        int32_t done = 0;
        CK(cudaMemcpyAsync(&done, &m->d_ctrl->done, sizeof done, cudaMemcpyDeviceToHost, m->stream));
        CK(cudaStreamSynchronize(m->stream));
        if (done) break;
    }
    return MB_OK;
}

/* Enqueues one CG solve (initial residual from V*, then iterations). */
static int cg_enqueue(mb_monodomain *m) {
    if (m->use_pcg) {
        CKK(pcg_launch(&m->pcg, m->stream));
        return MB_OK;
    }
    if (m->use_graphs) {
        CK(cudaGraphLaunch(m->ge_cg, m->stream));
        return MB_OK;
    }
    return cg_host_loop(m);
}

static int step_once(mb_monodomain *m) {
    if (m->use_graphs) {
        CK(cudaGraphLaunch(m->ge_step, m->stream));
        return MB_OK;
    }
    CKK(step_ode(m));
    int rc = cg_enqueue(m);
    if (rc) return rc;
    CKK(mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream));
    return MB_OK;
}

int mb_monodomain_step(mb_monodomain *m, int n) {
    if (!m || n < 0) return set_err(MB_ERR_ARG, "bad arguments");
    if (m->phase != 0) return set_err(MB_ERR_STATE, "a split step is in progress");
    for (int i = 0; i < n; ++i) {
        int rc = step_once(m);
        if (rc) return rc;
    }
    return MB_OK;
}

int mb_monodomain_sync(mb_monodomain *m) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    CK(cudaStreamSynchronize(m->stream));
    int32_t nan_flag = 0;
    CK(cudaMemcpy(&nan_flag, &m->d_ctrl->nan_flag, sizeof nan_flag, cudaMemcpyDeviceToHost));
    if (m->d_status) {
        int st = 0;
        CK(cudaMemcpy(&st, m->d_status, sizeof st, cudaMemcpyDeviceToHost));
        if (st) return set_err(MB_ERR_CUDA, "CG grid barrier timed out (status %d)", st);
    }
    if (nan_flag) return set_err(MB_ERR_NAN, "NaN in the CG error: the cell model diverged");
    if (m->ode.adaptive) {
        uint32_t unfinished = 0;
        CK(cudaMemcpy(&unfinished, &m->d_ctrl->ode_unfinished, sizeof unfinished, cudaMemcpyDeviceToHost));
        if (unfinished)
            return set_err(MB_ERR_NAN, "adaptive ODE step: %u cell steps did not reach the step's end time within "
                                       "the pass limit", unfinished);
    }
    return MB_OK;
}

/* ---- split API (the reference loop body one call at a time) ------------- */

int mb_solve_all_volumes_odes(mb_monodomain *m) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (m->phase != 0) return set_err(MB_ERR_STATE, "ODE step already taken for this time step");
    CKK(step_ode(m));
    m->phase = 1;
    return MB_OK;
}

/* b = alpha V* is formed inside the first CG kernel; this call only checks
 * the order of the phases. */
int mb_update_monodomain_default(mb_monodomain *m) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (m->phase != 1) return set_err(MB_ERR_STATE, "update_monodomain before the ODE step");
    m->phase = 2;
    return MB_OK;
}

int mb_conjugate_gradient(mb_monodomain *m, uint32_t *its, double *error) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (m->phase != 2) return set_err(MB_ERR_STATE, "conjugate_gradient before update_monodomain");
    {
        int rc = cg_enqueue(m);
        if (rc) return rc;
    }
    mb_ctrl c;
    CK(cudaMemcpyAsync(&c, m->d_ctrl, sizeof c, cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    if (its) *its = (uint32_t)c.its;
    if (error) *error = c.error;
    m->phase = 3;
    return MB_OK;
}

int mb_advance_time(mb_monodomain *m) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (m->phase != 3) return set_err(MB_ERR_STATE, "advance_time before conjugate_gradient");
    CKK(mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream));
    m->phase = 0;
    return MB_OK;
}

int mb_monodomain_step_host(mb_monodomain *m, const double *stim_host, double *v_host) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    mb_ode_dev o = m->ode;
    if (stim_host) {
        CK(cudaMemcpyAsync(m->d_stim_host, stim_host, (size_t)m->n_active * sizeof(double), cudaMemcpyHostToDevice,
                           m->stream));
        o.stim_host = m->d_stim_host;
    }
    if (m->use_ecg) CKK(mbk_ecg(&m->st, m->d_v, &m->ecg, m->d_ctrl, m->stream));
    CKK(mbk_ode_step(&o, m->d_ctrl, m->d_v, m->d_vstar, m->stream));
    {
        int rc = cg_enqueue(m);
        if (rc) return rc;
    }
    CKK(mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream));
    if (v_host) {
        CK(cudaMemcpyAsync(v_host, m->d_v, (size_t)m->n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        CK(cudaStreamSynchronize(m->stream));
    }
    return MB_OK;
}

/* Pipelined form of mb_monodomain_step_host.  Call k uses slot k % 2: the
 * stimulus is copied into the slot's device buffer on the host-to-device
 * stream (after the ODE of call k - 2 has read that buffer) while step k - 1
 * still runs, the step runs on the tissue's stream, V is snapshotted into
 * the slot's device buffer and copied to v_host on the device-to-host stream
 * while the next step runs; the two directions do not queue behind each
 * other.  The call returns once
 * the copies of call k - 1 are complete (its V is in its host buffer and its
 * buffers may be refilled), so the caller alternates two pairs of host
 * buffers (pinned memory for the copies to overlap); the last call's copies
 * are complete after mb_monodomain_host_wait. */
static int host_pipeline_init(mb_monodomain *m) {
    if (m->copy_stream) return MB_OK;
    const size_t sb = (size_t)m->n_active * sizeof(double), vb = (size_t)m->n * sizeof(double);
    cudaError_t e = cudaStreamCreateWithFlags(&m->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->h2d_stream, cudaStreamNonBlocking);
    for (int j = 0; j < 2 && e == cudaSuccess; ++j) {
        e = cudaMalloc((void **)&m->d_stim2[j], sb ? sb : 8);
        if (e == cudaSuccess) e = cudaMalloc((void **)&m->d_vsnap[j], vb);
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&m->hev[i][j], cudaEventDisableTiming);
        /* every slot starts free: record its events once */
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventRecord(m->hev[i][j], m->copy_stream);
    }
    if (e != cudaSuccess) return set_err(MB_ERR_CUDA, "host pipeline: %s", cudaGetErrorString(e));
    return MB_OK;
}

enum { HEV_STIM = 0, HEV_ODE = 1, HEV_VREADY = 2, HEV_VDONE = 3 };

int mb_monodomain_step_host_async(mb_monodomain *m, const double *stim_host, double *v_host) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    int rc = host_pipeline_init(m);
    if (rc) return rc;
    const int s = (int)(m->host_calls & 1);
    /* slot s was last used by call k - 2, whose copies call k - 1 waited for */
    mb_ode_dev o = m->ode;
    if (stim_host) {
        CK(cudaStreamWaitEvent(m->h2d_stream, m->hev[HEV_ODE][s], 0));
        CK(cudaMemcpyAsync(m->d_stim2[s], stim_host, (size_t)m->n_active * sizeof(double), cudaMemcpyHostToDevice,
                           m->h2d_stream));
        CK(cudaEventRecord(m->hev[HEV_STIM][s], m->h2d_stream));
        CK(cudaStreamWaitEvent(m->stream, m->hev[HEV_STIM][s], 0));
        o.stim_host = m->d_stim2[s];
    }
    if (m->use_ecg) CKK(mbk_ecg(&m->st, m->d_v, &m->ecg, m->d_ctrl, m->stream));
    CKK(mbk_ode_step(&o, m->d_ctrl, m->d_v, m->d_vstar, m->stream));
    CK(cudaEventRecord(m->hev[HEV_ODE][s], m->stream));
    rc = cg_enqueue(m);
    if (rc) return rc;
    CKK(mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream));
    if (v_host) {
        CK(cudaMemcpyAsync(m->d_vsnap[s], m->d_v, (size_t)m->n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
        CK(cudaEventRecord(m->hev[HEV_VREADY][s], m->stream));
        CK(cudaStreamWaitEvent(m->copy_stream, m->hev[HEV_VREADY][s], 0));
        CK(cudaMemcpyAsync(v_host, m->d_vsnap[s], (size_t)m->n * sizeof(double), cudaMemcpyDeviceToHost,
                           m->copy_stream));
    }
    CK(cudaEventRecord(m->hev[HEV_VDONE][s], m->copy_stream));
    m->host_calls += 1;
    /* the copies of call k - 1 (they ran under this step's compute) */
    CK(cudaEventSynchronize(m->hev[HEV_VDONE][1 - s]));
    return MB_OK;
}

int mb_monodomain_host_wait(mb_monodomain *m) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (m->copy_stream) CK(cudaStreamSynchronize(m->copy_stream));
    if (m->h2d_stream) CK(cudaStreamSynchronize(m->h2d_stream));
    CK(cudaStreamSynchronize(m->stream));
    return MB_OK;
}

/* n pipelined host-buffer steps alternating the two buffer pairs, timed from
 * before the first copy to after the last copy (CUDA events on both streams). */
int mb_monodomain_time_steps_host_async(mb_monodomain *m, int n, const double *stim0, const double *stim1,
                                        double *v0, double *v1, double *ms) {
    if (!m || n <= 0 || !ms) return set_err(MB_ERR_ARG, "bad arguments");
    int rc = host_pipeline_init(m);
    if (rc) return rc;
    CK(cudaStreamSynchronize(m->copy_stream));
    CK(cudaStreamSynchronize(m->h2d_stream));
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaEventRecord(m->ev[2], m->stream));
    CK(cudaStreamWaitEvent(m->copy_stream, m->ev[2], 0));
    CK(cudaStreamWaitEvent(m->h2d_stream, m->ev[2], 0));
    for (int i = 0; i < n; ++i) {
        const int s = (int)(m->host_calls & 1);
        rc = mb_monodomain_step_host_async(m, s ? stim1 : stim0, s ? v1 : v0);
        if (rc) return rc;
    }
    CK(cudaEventRecord(m->hev[HEV_VDONE][0], m->copy_stream));
    CK(cudaStreamWaitEvent(m->stream, m->hev[HEV_VDONE][0], 0));
    CK(cudaEventRecord(m->ev[3], m->stream));
    CK(cudaEventSynchronize(m->ev[3]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, m->ev[2], m->ev[3]));
    *ms = t;
    return MB_OK;
}

/* ---- state access --------------------------------------------------------- */

int mb_monodomain_get_v(mb_monodomain *m, double *v_host) {
    if (!m || !v_host) return set_err(MB_ERR_ARG, "null");
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaMemcpy(v_host, m->d_v, (size_t)m->n * sizeof(double), cudaMemcpyDeviceToHost));
    if (m->desc.active)
        for (int64_t g = 0; g < m->n; ++g) if (!m->desc.active[g]) v_host[g] = NAN;
    return MB_OK;
}

int mb_monodomain_set_v(mb_monodomain *m, const double *v_host) {
    if (!m || !v_host) return set_err(MB_ERR_ARG, "null");
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaMemcpy(m->d_v, v_host, (size_t)m->n * sizeof(double), cudaMemcpyHostToDevice));
    forget_stored_product(m);
    CK(cudaStreamSynchronize(m->stream));
    return MB_OK;
}

int mb_monodomain_get_state(mb_monodomain *m, double *state_host) {
    if (!m || !state_host) return set_err(MB_ERR_ARG, "null");
    double *d = NULL;
    const size_t bytes = (size_t)m->neq * m->n_active * sizeof(double);
    CK(cudaMalloc((void **)&d, bytes));
    /* V of the state is the grid V (after the CG) */
    CKK(mbk_ode_gather(&m->ode, m->d_v, d, m->stream));
    CK(cudaMemcpyAsync(state_host, d, bytes, cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    cudaFree(d);
    return MB_OK;
}

int mb_monodomain_get_ecg(mb_monodomain *m, int64_t first, int64_t n, double *times, double *values,
                          int64_t *records) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (!m->use_ecg) return set_err(MB_ERR_STATE, "the ECG is off (ecg_rate = 0)");
    mb_ctrl c;
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaMemcpy(&c, m->d_ctrl, sizeof c, cudaMemcpyDeviceToHost));
    if (records) *records = c.ecg_count;
    if (n <= 0) return MB_OK;
    if (first < 0 || first + n > c.ecg_count)
        return set_err(MB_ERR_ARG, "ECG records %lld..%lld requested, %lld taken", (long long)first,
                       (long long)(first + n - 1), (long long)c.ecg_count);
    const int nl = m->ecg.n_leads;
    const size_t row = (size_t)(1 + nl);
    double *tmp = (double *)malloc((size_t)n * row * sizeof(double));
    if (!tmp) return set_err(MB_ERR_NOMEM, "host memory");
    cudaError_t e = cudaMemcpy(tmp, m->d_ecg_log + (size_t)first * row, (size_t)n * row * sizeof(double),
                               cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        for (int64_t r = 0; r < n; ++r) {
            if (times) times[r] = tmp[(size_t)r * row];
            if (values)
                for (int l = 0; l < nl; ++l) values[(size_t)r * nl + l] = tmp[(size_t)r * row + 1 + l];
        }
    free(tmp);
    return e == cudaSuccess ? MB_OK : set_err(MB_ERR_CUDA, "ECG read-back: %s", cudaGetErrorString(e));
}

int mb_monodomain_get_activation(mb_monodomain *m, float *first, float *last, float *apd90, int32_t *count) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (!m->d_act) return set_err(MB_ERR_STATE, "activation tracking is off (track_activation = 0)");
    const size_t ld = m->ode.ld;
    float *h = (float *)malloc((size_t)MB_ACT_ROWS * ld * sizeof(float));
    if (!h) return set_err(MB_ERR_NOMEM, "host memory");
    cudaError_t e = cudaStreamSynchronize(m->stream);
    if (e == cudaSuccess) e = cudaMemcpy(h, m->d_act, (size_t)MB_ACT_ROWS * ld * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { free(h); return set_err(MB_ERR_CUDA, "%s", cudaGetErrorString(e)); }
    uint32_t t = 0;
    for (int64_t g = 0; g < m->n; ++g) {
        const int on = !m->h_mask || m->h_mask[g];
        const int st = on ? (int)h[MB_ACT_STATE * ld + t] : 0;
        if (first) first[g] = on ? h[MB_ACT_FIRST * ld + t] : -1.0f;
        if (last) last[g] = on ? h[MB_ACT_LAST * ld + t] : -1.0f;
        if (apd90) apd90[g] = on ? h[MB_ACT_APD * ld + t] : -1.0f;
        if (count) count[g] = st >> 1;
        if (on) ++t;
    }
    free(h);
    return MB_OK;
}

int mb_monodomain_info(mb_monodomain *m, int64_t *count, double *cur_time, uint32_t *n_active, int *neq) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    mb_ctrl c;
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaMemcpy(&c, m->d_ctrl, sizeof c, cudaMemcpyDeviceToHost));
    if (count) *count = c.count;
    if (cur_time) *cur_time = c.cur_time;
    if (n_active) *n_active = m->n_active;
    if (neq) *neq = m->neq;
    return MB_OK;
}

int mb_monodomain_step_stats(mb_monodomain *m, int64_t first, int64_t n, mb_step_stats *out) {
    if (!m || !out || first < 0 || n < 0 || first + n > m->log_len) return set_err(MB_ERR_ARG, "bad range");
    CK(cudaStreamSynchronize(m->stream));
    CK(cudaMemcpy(out, m->d_log + first, (size_t)n * sizeof(mb_step_stats), cudaMemcpyDeviceToHost));
    return MB_OK;
}

int mb_monodomain_device_v(mb_monodomain *m, double **v_dev, void **stream) {
    if (!m) return set_err(MB_ERR_ARG, "null");
    if (v_dev) *v_dev = m->d_v;
    if (stream) *stream = (void *)m->stream;
    return MB_OK;
}

/* Times n steps phase by phase with events on the launching stream: the ODE
 * kernel alone and the CG solve (initial residual + WHILE loop) alone. */
/* Device time of n whole steps, CUDA events on the tissue's stream. */
int mb_monodomain_time_steps(mb_monodomain *m, int n, double *ms) {
    if (!m || n <= 0 || !ms) return set_err(MB_ERR_ARG, "bad arguments");
    CK(cudaEventRecord(m->ev[0], m->stream));
    int rc = mb_monodomain_step(m, n);
    if (rc) return rc;
    CK(cudaEventRecord(m->ev[1], m->stream));
    CK(cudaEventSynchronize(m->ev[1]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, m->ev[0], m->ev[1]));
    *ms = t;
    return MB_OK;
}

/* Device time of n reference-host steps (stimulus H2D, ODE, CG, V D2H). */
int mb_monodomain_time_steps_host(mb_monodomain *m, int n, const double *stim_host, double *v_host, double *ms) {
    if (!m || n <= 0 || !ms) return set_err(MB_ERR_ARG, "bad arguments");
    CK(cudaEventRecord(m->ev[2], m->stream));
    for (int i = 0; i < n; ++i) {
        int rc = mb_monodomain_step_host(m, stim_host, v_host);
        if (rc) return rc;
    }
    CK(cudaEventRecord(m->ev[3], m->stream));
    CK(cudaEventSynchronize(m->ev[3]));
    float t = 0;
    CK(cudaEventElapsedTime(&t, m->ev[2], m->ev[3]));
    *ms = t;
    return MB_OK;
}

int mb_monodomain_profile_steps(mb_monodomain *m, int n, double *ode_ms, double *cg_ms, double *step_ms,
                                int *cg_iterations) {
    if (!m || n <= 0) return set_err(MB_ERR_ARG, "bad arguments");
    double to = 0, tc = 0, ts = 0;
    long its = 0;
    for (int i = 0; i < n; ++i) {
        CK(cudaEventRecord(m->ev[0], m->stream));
        CKK(step_ode(m));
        CK(cudaEventRecord(m->ev[1], m->stream));
        {
            int rc = cg_enqueue(m);
            if (rc) return rc;
        }
        CK(cudaEventRecord(m->ev[2], m->stream));
        CKK(mbk_step_end(m->d_ctrl, m->desc.dt_pde, m->desc.dt_ode, m->num_steps, m->d_log, m->log_len, m->stream));
        CK(cudaEventRecord(m->ev[3], m->stream));
        CK(cudaEventSynchronize(m->ev[3]));
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, m->ev[0], m->ev[1]);
        cudaEventElapsedTime(&b, m->ev[1], m->ev[2]);
        cudaEventElapsedTime(&c, m->ev[0], m->ev[3]);
        to += a; tc += b; ts += c;
        int32_t it = 0;
        cudaMemcpy(&it, &m->d_ctrl->its, sizeof it, cudaMemcpyDeviceToHost);
        its += it;
    }
    if (ode_ms) *ode_ms = to / n;
    if (cg_ms) *cg_ms = tc / n;
    if (step_ms) *step_ms = ts / n;
    if (cg_iterations) *cg_iterations = (int)(its / n);
    return MB_OK;
}

/* ---- general CSR CG -------------------------------------------------------- */

/* A CSR system kept on the device between solves (the reference-host shim
 * uploads the assembled matrix once and solves every step). */
struct mb_csr {
    mb_csr_dev a;
    int32_t *d_rp, *d_col;
    double *d_val, *d_b, *d_x, *d_r, *d_p, *d_q, *d_id, *d_part;
    mb_ctrl *d_ctrl;
    cudaStream_t s;
};

void mb_csr_destroy(mb_csr *m) {
    if (!m) return;
    if (m->s) cudaStreamSynchronize(m->s);
    void *bufs[] = {m->d_rp, m->d_col, m->d_val, m->d_b, m->d_x, m->d_r, m->d_p, m->d_q, m->d_id, m->d_part, m->d_ctrl};
    for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; ++i) cudaFree(bufs[i]);
    if (m->s) cudaStreamDestroy(m->s);
    free(m);
}

int mb_csr_create(mb_csr **out, int32_t n, const int32_t *row_ptr, const int32_t *col, const double *val) {
    if (!out || n <= 0 || !row_ptr || !col || !val) return set_err(MB_ERR_ARG, "bad arguments");
    const int32_t nnz = row_ptr[n];
    if (nnz < 0) return set_err(MB_ERR_ARG, "bad row_ptr");
    mb_csr *m = (mb_csr *)calloc(1, sizeof *m);
    if (!m) return set_err(MB_ERR_NOMEM, "out of host memory");
    int gb = (n + 255) / 256;
    if (gb > mbk_max_grid_blocks()) gb = mbk_max_grid_blocks();
    cudaError_t e = cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking);
#define CSR_ALLOC(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    CSR_ALLOC(m->d_rp, (size_t)(n + 1) * sizeof(int32_t));
    CSR_ALLOC(m->d_col, (size_t)(nnz ? nnz : 1) * sizeof(int32_t));
    CSR_ALLOC(m->d_val, (size_t)(nnz ? nnz : 1) * sizeof(double));
    CSR_ALLOC(m->d_b, (size_t)n * sizeof(double));
    CSR_ALLOC(m->d_x, (size_t)n * sizeof(double));
    CSR_ALLOC(m->d_r, (size_t)n * sizeof(double));
    CSR_ALLOC(m->d_p, (size_t)n * sizeof(double));
    CSR_ALLOC(m->d_q, (size_t)n * sizeof(double));
    CSR_ALLOC(m->d_id, (size_t)n * sizeof(double));
    CSR_ALLOC(m->d_part, (size_t)3 * gb * sizeof(double));
    CSR_ALLOC(m->d_ctrl, sizeof(mb_ctrl));
#undef CSR_ALLOC
    if (e == cudaSuccess) e = cudaMemcpy(m->d_rp, row_ptr, (size_t)(n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnz) e = cudaMemcpy(m->d_col, col, (size_t)nnz * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nnz) e = cudaMemcpy(m->d_val, val, (size_t)nnz * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        mb_csr_destroy(m);
        return set_err(MB_ERR_CUDA, "mb_csr_create: %s", cudaGetErrorString(e));
    }
    mb_csr_dev *a = &m->a;
    a->n = n;
    a->grid_blocks = gb;
    a->row_ptr = m->d_rp; a->col = m->d_col; a->val = m->d_val; a->b = m->d_b; a->x = m->d_x;
    a->r = m->d_r; a->p = m->d_p; a->q = m->d_q; a->inv_diag = m->d_id; a->partials = m->d_part;
    *out = m;
    return MB_OK;
}

int mb_csr_solve(mb_csr *m, const double *b, double *x, double tolerance, int max_iterations,
                 int use_preconditioner, uint32_t *number_of_iterations, double *error) {
    if (!m || !b || !x) return set_err(MB_ERR_ARG, "bad arguments");
    const size_t bytes = (size_t)m->a.n * sizeof(double);
    CK(cudaMemcpyAsync(m->d_b, b, bytes, cudaMemcpyHostToDevice, m->s));
    CK(cudaMemcpyAsync(m->d_x, x, bytes, cudaMemcpyHostToDevice, m->s));
    mb_ctrl c;
    memset(&c, 0, sizeof c);
    c.tol = tolerance;
    c.max_its = max_iterations;
    c.use_precond = use_preconditioner ? 1 : 0;
    CK(cudaMemcpyAsync(m->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice, m->s));
    if (mbk_csr_cg_init(&m->a, m->d_ctrl, m->s)) return set_err(MB_ERR_CUDA, "csr init launch failed");
    for (int it = 0; it < max_iterations + 1; it += 16) {
        for (int q = 0; q < 16; ++q)
            if (mbk_csr_cg_iter(&m->a, m->d_ctrl, m->s)) return set_err(MB_ERR_CUDA, "csr iteration launch failed");
        int32_t done = 0;
        CK(cudaMemcpyAsync(&done, &m->d_ctrl->done, sizeof done, cudaMemcpyDeviceToHost, m->s));
        CK(cudaStreamSynchronize(m->s));
        if (done) break;
    }
    CK(cudaMemcpyAsync(&c, m->d_ctrl, sizeof c, cudaMemcpyDeviceToHost, m->s));
    CK(cudaMemcpyAsync(x, m->d_x, bytes, cudaMemcpyDeviceToHost, m->s));
    CK(cudaStreamSynchronize(m->s));
    if (number_of_iterations) *number_of_iterations = (uint32_t)c.its;
    if (error) *error = c.error;
    return MB_OK;
}

int mb_csr_conjugate_gradient(int32_t n, const int32_t *row_ptr, const int32_t *col, const double *val,
                              const double *b, double *x, double tolerance, int max_iterations,
                              int use_preconditioner, uint32_t *number_of_iterations, double *error) {
    if (n <= 0 || !row_ptr || !col || !val || !b || !x) return set_err(MB_ERR_ARG, "bad arguments");
    mb_csr *m = NULL;
    int rc = mb_csr_create(&m, n, row_ptr, col, val);
    if (rc) return rc;
    rc = mb_csr_solve(m, b, x, tolerance, max_iterations, use_preconditioner, number_of_iterations, error);
    mb_csr_destroy(m);
    return rc;
}

/* ---- internals used by the adjoint ----------------------------------------- */

int mb_internal_error(int code, const char *msg) { return set_err(code, "%s", msg); }

static size_t align256(size_t b) { return (b + 255u) & ~(size_t)255u; }

/* snapshot layout: V | V* | FP64 state rows | FP32 state rows | control block */
static void snapshot_layout(const mb_monodomain *m, size_t off[5], size_t len[5]) {
    int n64, n32;
    ode_rows(m->desc.model, m->desc.precision, m->desc.ode_adaptive, &n64, &n32);
    len[0] = (size_t)m->n * sizeof(double);
    len[1] = (size_t)m->n * sizeof(double);
    len[2] = (size_t)n64 * m->ode.ld * sizeof(double);
    len[3] = (size_t)n32 * m->ode.ld * sizeof(float);
    len[4] = sizeof(mb_ctrl);
    size_t o = 0;
    for (int q = 0; q < 5; ++q) {
        off[q] = o;
        o += align256(len[q]);
    }
}

size_t mb_tissue_snapshot_bytes(const mb_monodomain *m) {
    size_t off[5], len[5];
    snapshot_layout(m, off, len);
    return off[4] + align256(len[4]);
}

int mb_tissue_snapshot(mb_monodomain *m, void *dev, int restore) {
    size_t off[5], len[5];
    snapshot_layout(m, off, len);
    void *live[5] = {m->d_v, m->d_vstar, m->d_sv64, m->d_sv32, m->d_ctrl};
    for (int q = 0; q < 5; ++q) {
        if (!len[q] || !live[q]) continue;
        char *snap = (char *)dev + off[q];
        cudaError_t e = restore ? cudaMemcpyAsync(live[q], snap, len[q], cudaMemcpyDeviceToDevice, m->stream)
                                : cudaMemcpyAsync(snap, live[q], len[q], cudaMemcpyDeviceToDevice, m->stream);
        if (e != cudaSuccess) return set_err(MB_ERR_CUDA, "snapshot copy: %s", cudaGetErrorString(e));
    }
    if (restore) forget_stored_product(m);
    return MB_OK;
}

void mb_tissue_snapshot_parts(const mb_monodomain *m, void *dev, double **v, double **sv64, mb_ctrl **ctrl) {
    size_t off[5], len[5];
    snapshot_layout(m, off, len);
    if (v) *v = (double *)((char *)dev + off[0]);
    if (sv64) *sv64 = (double *)((char *)dev + off[2]);
    if (ctrl) *ctrl = (mb_ctrl *)((char *)dev + off[4]);
}

float *mb_tissue_snapshot_sv32(const mb_monodomain *m, void *dev) {
    size_t off[5], len[5];
    snapshot_layout(m, off, len);
    return len[3] ? (float *)((char *)dev + off[3]) : NULL;
}

int mb_tissue_set_sigma(mb_monodomain *m, const double *sigma_cell) {
    if (!m || !sigma_cell || m->desc.assembly != MB_ASSEMBLY_PER_CELL_SIGMA || !m->d_fx)
        return set_err(MB_ERR_ARG, "new conductivities need a per-cell-sigma tissue");
    mb_monodomain_desc d = m->desc;
    d.sigma_cell = sigma_cell;
    mb_assembly_out a;
    int rc = mb_assemble(&d, &a);
    if (rc) { mb_assembly_free(&a); return set_err(rc, "assembly failed"); }
    const size_t bytes = (size_t)m->n * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(m->d_fx, a.fx, bytes, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_fy, a.fy, bytes, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_fz, a.fz, bytes, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    mb_assembly_free(&a);
    if (e != cudaSuccess) return set_err(MB_ERR_CUDA, "%s", cudaGetErrorString(e));
    if (m->use_pcg) CKK(mbk_inv_diag(&m->st, m->d_invd, m->d_invd32, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    return MB_OK;
}

int mb_tissue_set_scale(mb_monodomain *m, const double *scale) {
    if (!m || !scale || !m->d_scale) return set_err(MB_ERR_ARG, "new scalings need a tissue created with scalings");
    const size_t ld = m->ode.ld;
    float *h = (float *)calloc((size_t)MB_NUM_SCALES * ld, sizeof(float));
    if (!h) return set_err(MB_ERR_NOMEM, "host memory");
    uint32_t t = 0;
    for (int64_t g = 0; g < m->n; ++g) {
        if (m->h_mask && !m->h_mask[g]) continue;
        for (int q = 0; q < MB_NUM_SCALES; ++q) h[(size_t)q * ld + t] = (float)scale[(size_t)q * m->n + g];
        ++t;
    }
    cudaError_t e = cudaMemcpy(m->d_scale, h, (size_t)MB_NUM_SCALES * ld * sizeof(float), cudaMemcpyHostToDevice);
    free(h);
    if (e != cudaSuccess) return set_err(MB_ERR_CUDA, "%s", cudaGetErrorString(e));
    return MB_OK;
}

/* ---- checkpoints and V files ------------------------------------------------- */

typedef struct ckpt_header {
    char magic[8];          /* "MBCKPT1" */
    int32_t nx, ny, nz, model, precision, has_act;
    uint64_t n_active, ld, snap_bytes, act_bytes;
} ckpt_header;

int mb_monodomain_checkpoint_bytes(mb_monodomain *m, size_t *bytes) {
    if (!m || !bytes) return set_err(MB_ERR_ARG, "null");
    const size_t act = m->d_act ? (size_t)MB_ACT_ROWS * m->ode.ld * sizeof(float) : 0;
    *bytes = align256(sizeof(ckpt_header)) + mb_tissue_snapshot_bytes(m) + act;
    return MB_OK;
}

static int ckpt_copy(mb_monodomain *m, char *host, int restore) {
    size_t off[5], len[5];
    snapshot_layout(m, off, len);
    const size_t base = align256(sizeof(ckpt_header));
    void *live[5] = {m->d_v, m->d_vstar, m->d_sv64, m->d_sv32, m->d_ctrl};
    CK(cudaStreamSynchronize(m->stream));
    for (int q = 0; q < 5; ++q) {
        if (!len[q] || !live[q]) continue;
        if (restore) CK(cudaMemcpy(live[q], host + base + off[q], len[q], cudaMemcpyHostToDevice));
        else CK(cudaMemcpy(host + base + off[q], live[q], len[q], cudaMemcpyDeviceToHost));
    }
    if (m->d_act) {
        const size_t abytes = (size_t)MB_ACT_ROWS * m->ode.ld * sizeof(float);
        char *p = host + base + mb_tissue_snapshot_bytes(m);
        if (restore) CK(cudaMemcpy(m->d_act, p, abytes, cudaMemcpyHostToDevice));
        else CK(cudaMemcpy(p, m->d_act, abytes, cudaMemcpyDeviceToHost));
    }
    if (restore) {
        forget_stored_product(m);
        CK(cudaStreamSynchronize(m->stream));
    }
    return MB_OK;
}

int mb_monodomain_checkpoint(mb_monodomain *m, void *host, size_t bytes) {
    size_t need = 0;
    int rc = mb_monodomain_checkpoint_bytes(m, &need);
    if (rc) return rc;
    if (!host || bytes < need) return set_err(MB_ERR_ARG, "checkpoint buffer smaller than %zu bytes", need);
    if (m->phase != 0) return set_err(MB_ERR_STATE, "a split step is in progress");
    ckpt_header h;
    memset(&h, 0, sizeof h);
    memcpy(h.magic, "MBCKPT1", 8);
    h.nx = m->desc.nx; h.ny = m->desc.ny; h.nz = m->desc.nz;
    h.model = m->desc.model; h.precision = m->desc.precision; h.has_act = m->d_act != NULL;
    h.n_active = m->n_active; h.ld = m->ode.ld; h.snap_bytes = mb_tissue_snapshot_bytes(m);
    h.act_bytes = m->d_act ? (uint64_t)MB_ACT_ROWS * m->ode.ld * sizeof(float) : 0;
    memcpy(host, &h, sizeof h);
    return ckpt_copy(m, (char *)host, 0);
}

int mb_monodomain_restore(mb_monodomain *m, const void *host, size_t bytes) {
    size_t need = 0;
    int rc = mb_monodomain_checkpoint_bytes(m, &need);
    if (rc) return rc;
    if (!host || bytes < need) return set_err(MB_ERR_ARG, "checkpoint buffer smaller than %zu bytes", need);
    if (m->phase != 0) return set_err(MB_ERR_STATE, "a split step is in progress");
    ckpt_header h;
    memcpy(&h, host, sizeof h);
    if (memcmp(h.magic, "MBCKPT1", 8) != 0 || h.nx != m->desc.nx || h.ny != m->desc.ny || h.nz != m->desc.nz ||
        h.model != m->desc.model || h.precision != m->desc.precision || h.n_active != m->n_active ||
        h.ld != m->ode.ld || h.snap_bytes != mb_tissue_snapshot_bytes(m) || h.has_act != (m->d_act != NULL))
        return set_err(MB_ERR_ARG, "checkpoint does not belong to a tissue of this shape, model and precision");
    return ckpt_copy(m, (char *)host, 1);
}

/* V of the active cells as save_as_text_or_binary writes it
 * (save_mesh.c:248-420): per cell the centre, half the cell size and V,
 * "%g,%g,%g,%g,%g,%g,%g\n" as text or 7 doubles as binary; cells in grid
 * order (the reference writes its own traversal order; match by centre). */
int mb_monodomain_save_v(mb_monodomain *m, const char *path, int binary) {
    if (!m || !path) return set_err(MB_ERR_ARG, "null");
    double *v = (double *)malloc((size_t)m->n * sizeof(double));
    if (!v) return set_err(MB_ERR_NOMEM, "host memory");
    int rc = mb_monodomain_get_v(m, v);
    if (rc) { free(v); return rc; }
    FILE *f = fopen(path, binary ? "wb" : "w");
    if (!f) { free(v); return set_err(MB_ERR_ARG, "cannot open %s", path); }
    const mb_monodomain_desc *d = &m->desc;
    const double hx = d->dx / 2.0, hy = d->dy / 2.0, hz = d->dz / 2.0;
    for (int64_t g = 0; g < m->n; ++g) {
        if (m->h_mask && !m->h_mask[g]) continue;
        const int64_t i = g % d->nx, j = (g / d->nx) % d->ny, k = g / ((int64_t)d->nx * d->ny);
        const double rec[7] = {(i + 0.5) * d->dx, (j + 0.5) * d->dy, (k + 0.5) * d->dz, hx, hy, hz, v[g]};
        if (binary) fwrite(rec, sizeof(double), 7, f);
        else fprintf(f, "%g,%g,%g,%g,%g,%g,%g\n", rec[0], rec[1], rec[2], rec[3], rec[4], rec[5], rec[6]);
    }
    const int bad = ferror(f);
    fclose(f);
    free(v);
    return bad ? set_err(MB_ERR_ARG, "write to %s failed", path) : MB_OK;
}

/* Internal layout shared by the host driver (C) and the kernels (CUDA).
 * Nothing here is part of the public ABI. */
#ifndef MB_INTERNAL_H
#define MB_INTERNAL_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>
#include "monoalg3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MB_NEQ_TT2006 19
#define MB_NEQ_TORORD 43
#define MB_MAX_NEQ 43

/* Device-resident control block of one tissue: the loop clock, the stimulus
 * table and the scalars of the CG recurrences.  All of the per-step control
 * flow (stimulus windows, CG stopping rule, time advance) reads and writes
 * this block on the device, so a captured step never returns to the host. */
typedef struct mb_ctrl {
    /* loop clock (monodomain_solver.c:616,907-908) */
    double  cur_time;
    double  final_time;
    int64_t count;
    /* stimuli (ode_solver.c:201-235) */
    int32_t num_stims;
    int32_t nan_flag;
    double  stim_start[MB_MAX_STIMS];
    double  stim_dur[MB_MAX_STIMS];
    double  stim_period[MB_MAX_STIMS];
    double  stim_current[MB_MAX_STIMS];
    /* CG scalars (linear_system_solver.c:47-183) */
    double  rz, rr, pq, alpha, beta;
    double  rr_ref;          /* true r.r at the last refinement (mixed)    */
    double  error;
    double  tol;
    double  refine_ratio;
    double  refine_floor;    /* mixed: the FP32 recurrence runs down to at
                                least this r.r before the FP64 residual    */
    int32_t its;
    int32_t max_its;
    int32_t done;
    int32_t phase;           /* mixed: 1 = evaluate the FP64 true residual */
    int32_t refinements;
    int32_t use_precond;
    uint32_t ticket;
    uint32_t ode_unfinished; /* cells whose adaptive ODE step ran out of passes */
    /* activation tracking (ODE kernels) */
    double  act_dt;          /* loop step dt_pde                            */
    float   act_threshold;   /* upward crossing that marks an activation    */
    float   act_min_interval;/* ms between two counted activations          */
    /* pseudo-bidomain ECG */
    int64_t ecg_count;       /* records written                              */
    /* z-march fused CG: 1 while the product A x the last solve stored (the
     * tissue's zc_w) belongs to the current x; anything else that writes V
     * clears it (a stale product costs iterations, never the answer: the
     * stopping test is always on a residual from the stencil) */
    int32_t w_valid;
    int32_t pad_w_;
} mb_ctrl;

/* Structured grid, device view. */
typedef struct mb_grid_dev {
    int32_t nx, ny, nz, pad_;
    int64_t n;               /* nx*ny*nz                                    */
} mb_grid_dev;

/* 7-point operator (alpha I + K) on the structured grid.
 *   kind 0: constant face coefficients cx, cy, cz; mask gives removed cells
 *   kind 1: per-face coefficients fx, fy, fz stored at the lower cell
 *   kind 2: 27-point rows from a class table, class = (k, xy boundary kind) */
typedef struct mb_stencil_dev {
    int32_t kind;
    int32_t nx, ny, nz;
    double  alpha;
    double  cx, cy, cz;
    const uint8_t *mask;      /* NULL = all active                          */
    const double  *fx, *fy, *fz;
    const double  *table;     /* kind 2: [nz][9][27]                        */
    const float   *table32;   /* kind 2, FP32 copy                          */
    const uint8_t *code;      /* kinds 0, 1: per cell, bit q (q = 0..5 for
                                 -x,+x,-y,+y,-z,+z) = that neighbour couples,
                                 bit 6 = the cell is active                 */
    const uint16_t *rowid;    /* kind 2: per cell, k * 9 + class            */
    uint32_t nzmask;          /* kind 2: bit q = entry q is non-zero in some
                                 row of the table (bit 13, the diagonal,
                                 always set); entries whose bit is clear are
                                 zero in every row and are not read        */
} mb_stencil_dev;

/* ODE state, device view.  Rows of double (sv64) and float (sv32), each of
 * length ld; compact cell t lives at column t.  V is passed separately. */
typedef struct mb_ode_dev {
    int32_t model, precision, rl_rule, num_steps;
    uint32_t n;               /* cells to solve                             */
    uint32_t ld;              /* row stride (elements)                      */
    const uint32_t *cell;     /* compact -> grid index, NULL = identity     */
    double *sv64;
    float  *sv32;
    const uint8_t *stim_bits; /* per compact cell, bit k = stim config k    */
    const uint8_t *celltype;  /* per compact cell (ToRORd), NULL = endo     */
    const float   *scale;     /* MB_NUM_SCALES rows of ld, NULL = 1         */
    const double  *stim_host; /* per compact cell external stimulus, or NULL */
    double dt;
    int32_t variant;          /* register-budget variant chosen by the autotuner */
    uint32_t out_ld;          /* row stride of out64/out32                  */
    double *out64;            /* if set, the new state goes here (tuning)   */
    float  *out32;
    float  *act;              /* activation tracking, MB_ACT_ROWS rows of ld,
                                 NULL = off                                 */
    /* adaptive forward Euler (MB_MODEL_TORORD_FKATP_ENDO): 0 = fixed step;
       else sv64 rows NEQ..NEQ+2 hold each cell's dt, time_new, previous_dt
       and a loop step integrates to cur_time + adapt_span                  */
    int32_t adaptive;
    double min_dt, max_dt, abs_tol, rel_tol, adapt_span;
    double cur_time;          /* loop time when no control block is given   */
} mb_ode_dev;

/* Rows of the activation-tracking array (per compact cell). */
#define MB_ACT_VPREV 0        /* V at the previous loop step (NaN = none)   */
#define MB_ACT_FIRST 1        /* first activation time, ms (-1 = none)      */
#define MB_ACT_LAST 2         /* latest activation time, ms (-1 = none)     */
#define MB_ACT_APD 3          /* APD90 of the latest beat, ms (-1 = open)   */
#define MB_ACT_VPEAK 4        /* peak V since the latest activation         */
#define MB_ACT_VREST 5        /* lowest V since the last repolarisation     */
#define MB_ACT_STATE 6        /* 2 x activations + (1 while depolarised)    */
#define MB_ACT_ROWS 7

#define MB_ODE_VARIANTS 10    /* 0..5: one launch, min resident blocks of 128
                                 threads 1 .. 6; 6..9: staged persistent
                                 kernels, min resident blocks 1 .. 4 */
int mbk_ode_step_mixed(const mb_ode_dev *o, mb_ctrl *ctrl, const double *vin, double *vout,
                       cudaStream_t s);

/* ---- kernel launchers (kernels.cu) ------------------------------------ */
int mbk_ode_init(const mb_ode_dev *o, const double *table_dev, int ntypes, cudaStream_t s);
int mbk_ode_step(const mb_ode_dev *o, mb_ctrl *ctrl, const double *vin, double *vout,
                 cudaStream_t s);
int mbk_ode_gather(const mb_ode_dev *o, const double *v, double *out_dev, cudaStream_t s);
int mbk_ode_scatter(const mb_ode_dev *o, const double *in_dev, double *v, cudaStream_t s);

/* CG on the structured stencil.  FP64 vectors: r, p (double).  Mixed: r32, p32. */
typedef struct mb_cg_dev {
    int      precision;
    int      grid_blocks;
    double  *x;          /* V (solution), grid order                          */
    const double *vstar; /* V* after the ODEs; b = alpha * V*                 */
    double  *r, *p;      /* FP64 recurrences                                  */
    float   *r32, *p32;  /* FP32 recurrences (mixed)                          */
    double  *partials;   /* 2 * grid_blocks                                   */
    const double *b;     /* explicit right-hand side (CSR path) or NULL       */
} mb_cg_dev;

int mbk_cg_init(const mb_stencil_dev *st, const mb_cg_dev *cg, mb_ctrl *ctrl,
                unsigned long long cond, int use_cond, cudaStream_t s);
int mbk_cg_body(const mb_stencil_dev *st, const mb_cg_dev *cg, mb_ctrl *ctrl,
                unsigned long long cond, int use_cond, cudaStream_t s);
int mbk_step_end(mb_ctrl *ctrl, double dt_pde, double dt_ode, int num_steps,
                 mb_step_stats *log, int64_t log_len, cudaStream_t s);
int mbk_set_nan(double *v, const uint8_t *mask, int64_t n, cudaStream_t s);

/* CSR CG (general matrices). */
typedef struct mb_csr_dev {
    int32_t n;
    const int32_t *row_ptr, *col;
    const double *val;
    const double *b;
    double *x, *r, *p, *q, *inv_diag;
    double *partials;
    int grid_blocks;
} mb_csr_dev;
int mbk_csr_cg_init(const mb_csr_dev *a, mb_ctrl *ctrl, cudaStream_t s);
int mbk_csr_cg_iter(const mb_csr_dev *a, mb_ctrl *ctrl, cudaStream_t s);

int mbk_max_grid_blocks(void);

/* Persistent cooperative CG (one launch per solve). */
typedef struct mb_pcg_dev {
    mb_stencil_dev st;
    int mixed;
    int blocks;
    double *x;
    const double *vstar;
    const double *b;
    double *r64, *pa64, *pb64;
    float *r32, *pa32, *pb32;
    double *z64;             /* preconditioned residual (flat kernel)     */
    float *z32;
    double *ap64;            /* A p of the current direction (flat kernel) */
    float *ap32;
    float *ap32b;            /* second A p buffer (z-march fused pass, mixed) */
    const double *inv_diag64;/* Jacobi 1/diag (FP64 form)   */
    const float *inv_diag32; /* Jacobi 1/diag (mixed form)  */
    double *partials;        /* 2 * 8 * blocks + 16 */
    mb_ctrl *ctrl;
    unsigned *bar;           /* 2 words, zero at start */
    int *status;             /* 0 = ok; set on a barrier timeout */
    int form;                /* MB_PCG_FLAT, MB_PCG_TILED or MB_PCG_RESIDENT */
    int variant;             /* launch-shape variant of cg_flat.cu */
    int tiles_x, tiles_y, zchunk, nchunks;
    /* resident kernel (cg_resident.cu): shape, tile grid and tile size,
     * dynamic shared memory per block */
    int rc_shape, rc_nbx, rc_nby, rc_tw, rc_th;
    size_t rc_smem;
    double *rtrue;           /* resident kernel: FP64 true residual per cell */
    /* z-march kernel (cg_zmarch.cu): variant, per-plane Jacobi tables
     * (nz x 9 row classes) and the device array of its tensor maps */
    int zc_variant;
    double *zc_inv64;
    float *zc_inv32;
    float *zc_ptab32;       /* [nz][mbk_zcg_ptab_floats()] per-plane blocks (window Q pass) */
    double *zc_w;           /* A x of the fused solve's last residual (mixed), or NULL */
    void *zc_maps;
} mb_pcg_dev;
enum { MB_PCG_FLAT = 0, MB_PCG_TILED = 1, MB_PCG_RESIDENT = 2, MB_PCG_ZMARCH = 3 };
int mbk_fcg_variants(int kind);
int mbk_fcg_variant_groups(int variant);
int mbk_fcg_max_blocks(int mixed, int kind, int variant);
int mbk_fcg_launch(const mb_pcg_dev *p, cudaStream_t s);
int mbk_tcg_max_blocks(int mixed);
int mbk_tcg_launch(const mb_pcg_dev *p, cudaStream_t s);
void mbk_tcg_layout(int nx, int ny, int nz, int blocks, int *tiles_x, int *tiles_y, int *zchunk, int *nchunks);
int mbk_rcg_plan(mb_pcg_dev *p);
int mbk_rcg_launch(const mb_pcg_dev *p, cudaStream_t s);
int mbk_inv_diag(const mb_stencil_dev *st, double *d64, float *d32, cudaStream_t s);
int mbk_zcg_variants(void);
int mbk_zcg_max_blocks(int mixed, int variant);
int mbk_zcg_usable(const mb_stencil_dev *st);
int mbk_zcg_inv_tables(const mb_stencil_dev *st, double *inv64, float *inv32, float *ptab32, cudaStream_t s);
int mbk_zcg_ptab_floats(void);
int mbk_zcg_prepare(mb_pcg_dev *p);
int mbk_zcg_launch(const mb_pcg_dev *p, cudaStream_t s);

/* Pseudo-bidomain ECG at the start of a step (ecg.cu). */
typedef struct mb_ecg_dev {
    int32_t rate, n_leads;
    int64_t capacity;
    double dx, dy, dz, scale;  /* scale = 1 / (4 pi sigma_b) */
    const double *leads;       /* 3 x n_leads */
    double *partials;          /* MB_ECG_BLOCKS x MB_ECG_MAX_LEADS */
    double *log;               /* capacity x (1 + n_leads): time, leads */
} mb_ecg_dev;
#define MB_ECG_BLOCKS 296
int mbk_ecg(const mb_stencil_dev *st, const double *v, const mb_ecg_dev *e, mb_ctrl *ctrl, cudaStream_t s);
int mbk_stencil_codes(const mb_stencil_dev *st, uint8_t *code, uint16_t *rowid, cudaStream_t s);

#ifdef __cplusplus
}
#endif

#endif

/* The tissue object behind mb_monodomain (host, C), shared by the host
 * driver (monodomain.c) and the adjoint (adjoint.c).  Internal. */
#ifndef MB_TISSUE_H
#define MB_TISSUE_H

#include <stdint.h>
#include <cuda_runtime_api.h>
#include "mb_internal.h"

#ifdef __cplusplus
extern "C" {
#endif

struct mb_monodomain {
    mb_monodomain_desc desc;
    int neq;
    int num_steps;
    int64_t n;            /* grid cells */
    uint32_t n_active;
    cudaStream_t stream;

    uint8_t *d_mask;
    uint32_t *d_cells;
    double *d_v, *d_vstar;
    double *d_r, *d_p;
    float *d_r32, *d_p32;
    double *d_partials;
    double *d_sv64;
    float *d_sv32;
    uint8_t *d_stim_bits;
    uint8_t *d_celltype;
    float *d_scale;
    double *d_fx, *d_fy, *d_fz;
    double *d_table;
    float *d_table32;
    uint8_t *d_code;      /* per-cell coupling codes (kinds 0, 1) */
    uint16_t *d_rowid;    /* per-cell class-table rows (kind 2)   */
    float *d_act;         /* activation tracking rows, or NULL    */
    int use_ecg;          /* pseudo-bidomain ECG records at step starts */
    mb_ecg_dev ecg;
    double *d_ecg_leads, *d_ecg_part, *d_ecg_log;
    double *d_stim_host;
    mb_ctrl *d_ctrl;
    mb_step_stats *d_log;
    int64_t log_len;
    uint8_t *h_mask;      /* owned copy of desc.active (NULL = all active) */
    /* persistent CG */
    int use_pcg;
    mb_pcg_dev pcg;
    double *d_pb, *d_ppart, *d_invd, *d_z;
    float *d_pb32, *d_invd32, *d_z32;
    double *d_rtrue;             /* resident CG: FP64 true residual */
    double *d_ap;                /* flat CG: A p (FP64 form) */
    float *d_ap32;               /* flat CG: A p (mixed form) */
    float *d_ap32b;              /* z-march fused pass: second A p buffer (mixed form) */
    unsigned *d_bar;
    int *d_status;
    float cg_tune_ms;     /* device time of one CG solve of the chosen kernel at tuning */

    mb_ode_dev ode;
    mb_stencil_dev st;
    mb_cg_dev cg;

    cudaGraph_t g_pre, g_body_owner_unused, g_post;
    cudaGraph_t g_step;
    cudaGraphExec_t ge_step;
    cudaGraph_t g_cg;
    cudaGraphExec_t ge_cg;
    int use_graphs;
    int phase;            /* split-API state: 0 idle, 1 ODE done, 2 RHS formed */
    cudaEvent_t ev[4];
    /* pipelined host-buffer steps (mb_monodomain_step_host_async): one copy
     * stream per direction, two slots of device stimulus and V snapshot, and
     * per slot the events stimulus-copied, ODE-done (slot stimulus free),
     * V-snapshot-ready and V-copied (slot snapshot and host buffer free) */
    cudaStream_t copy_stream;     /* device -> host (V) */
    cudaStream_t h2d_stream;      /* host -> device (stimulus) */
    double *d_stim2[2], *d_vsnap[2];
    cudaEvent_t hev[4][2];
    int64_t host_calls;
};

/* Device-to-device snapshot of the loop state (V, V*, the ODE state rows and
 * the control block), for checkpoints: bytes needed, and save (restore = 0)
 * or restore (restore = 1) on the tissue's stream. */
size_t mb_tissue_snapshot_bytes(const mb_monodomain *m);
int mb_tissue_snapshot(mb_monodomain *m, void *dev, int restore);
/* Pointers into a snapshot: V, the FP64 state rows, the control block. */
void mb_tissue_snapshot_parts(const mb_monodomain *m, void *dev, double **v, double **sv64, mb_ctrl **ctrl);
/* The FP32 state rows of a snapshot (mixed precision; NULL otherwise). */
float *mb_tissue_snapshot_sv32(const mb_monodomain *m, void *dev);
/* New per-cell conductivity (grid order; PER_CELL_SIGMA tissues) and new
 * conductance scalings (MB_NUM_SCALES x grid; tissues created with them). */
int mb_tissue_set_sigma(mb_monodomain *m, const double *sigma_cell);
int mb_tissue_set_scale(mb_monodomain *m, const double *scale);
/* Records an error message for mb_last_error and returns code. */
int mb_internal_error(int code, const char *msg);

#ifdef __cplusplus
}
#endif
#endif

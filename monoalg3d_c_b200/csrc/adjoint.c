/* Discrete adjoint of the monodomain loop (host, C): gradients of a misfit
 * between simulated and observed V at sensor cells with respect to the
 * per-cell conductivity and the per-cell gKr scaling (ten Tusscher 2006,
 * per-cell conductivity, one Rush-Larsen sub-step per loop step), for the
 * FP64 forward or the mixed one (FP32 cell model and CG recurrences, FP64
 * V and concentrations): the mixed adjoint forms the cell model's Jacobian in
 * FP32, solves the transposed system with the mixed CG and accumulates every
 * adjoint vector and gradient in FP64.
 *
 * Forward: from the tissue's initial state, run nsteps loop steps, sampling V
 * at the sensor cells after every sample_every steps and storing a snapshot of
 * the loop state every checkpoint_every steps.
 * Backward: for each checkpoint segment, last first, restore its snapshot,
 * recompute the segment's states (kept on the device), then walk its steps
 * backwards: add the sampled gradients at the sensors, solve A w = lambda
 * with the tissue's persistent PCG, add the conductivity gradient of the
 * faces, and apply the transposed Jacobian of the Rush-Larsen step
 * (adjoint_kernels.cu).  The gradient sums are FP64.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "mb_internal.h"
#include "mb_tissue.h"

int mbk_adj_tt2006(const mb_ode_dev *o, const mb_ctrl *ctrl_n, const double *v_n, const double *sv_n,
                   const double *w, double alpha, const double *mu_in, double *mu_out, double *lam_out,
                   double *gth, cudaStream_t s);
int mbk_adj_tt2006_mixed(const mb_ode_dev *o, const mb_ctrl *ctrl_n, const double *v_n, const double *sv64_n,
                         const float *sv32_n, const double *w, double alpha, const double *mu_in, double *mu_out,
                         double *lam_out, double *gth, cudaStream_t s);
int mbk_adj_face_grad(const mb_stencil_dev *st, const double *sigma, const double *w, const double *v,
                      double mx, double my, double mz, double *gsig, cudaStream_t s);
int mbk_adj_gather(const double *v, const int64_t *cells, int ns, double *out, cudaStream_t s);
int mbk_adj_scatter(double *lam, const int64_t *cells, int ns, const double *gsrc, cudaStream_t s);
int mbk_adj_tol(const double *lam, int64_t n, double rel2, mb_ctrl *c, cudaStream_t s);

struct mb_adjoint {
    mb_monodomain *m;
    int nsteps, every, ns, sample_every, nsamples, nseg;
    int64_t *d_sensors;
    size_t snap;           /* bytes of one snapshot */
    char *d_ckpt;          /* nseg snapshots (the initial state first) */
    char *d_seg;           /* every + 1 snapshots of one segment */
    double *d_traces;      /* nsamples x ns */
    double *d_g;           /* nsamples x ns sampled gradients */
    double *d_lam, *d_lam2, *d_w, *d_mu, *d_mu2, *d_gsig, *d_gth, *d_sigma;
    mb_ctrl *d_actrl;      /* control block of the transposed solves */
    double alpha, mx, my, mz;
    int have_forward;
};

#define AERR(code, msg) mb_internal_error((code), (msg))
#define ACK(call)                                                              \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return AERR(MB_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)
#define AKK(call)                                                              \
    do {                                                                       \
        int e_ = (call);                                                       \
        if (e_ != 0) return AERR(MB_ERR_CUDA, cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

void mb_adjoint_destroy(mb_adjoint *a) {
    if (!a) return;
    void *bufs[] = {a->d_sensors, a->d_ckpt, a->d_seg, a->d_traces, a->d_g, a->d_lam, a->d_lam2, a->d_w, a->d_mu,
                    a->d_mu2, a->d_gsig, a->d_gth, a->d_sigma, a->d_actrl};
    for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; ++i) cudaFree(bufs[i]);
    mb_monodomain_destroy(a->m);
    free(a);
}

int mb_adjoint_create(mb_adjoint **out, const mb_monodomain_desc *d, int nsteps, int checkpoint_every,
                      int n_sensors, const int64_t *sensor_cells, int sample_every) {
    if (!out || !d || nsteps <= 0 || checkpoint_every <= 0 || n_sensors <= 0 || !sensor_cells || sample_every <= 0)
        return AERR(MB_ERR_ARG, "mb_adjoint_create: bad arguments");
    if (d->model != MB_MODEL_TT2006 || d->assembly != MB_ASSEMBLY_PER_CELL_SIGMA || !d->sigma_cell ||
        !d->current_scale || d->dt_ode != d->dt_pde)
        return AERR(MB_ERR_UNSUPPORTED, "the adjoint needs TT2006, per-cell sigma, conductance scalings and "
                                        "one ODE sub-step per loop step");
    const int64_t n = (int64_t)d->nx * d->ny * d->nz;
    for (int i = 0; i < n_sensors; ++i)
        if (sensor_cells[i] < 0 || sensor_cells[i] >= n || (d->active && !d->active[sensor_cells[i]]))
            return AERR(MB_ERR_ARG, "sensor outside the active cells");
    mb_adjoint *a = (mb_adjoint *)calloc(1, sizeof *a);
    if (!a) return AERR(MB_ERR_NOMEM, "host memory");
    int rc = mb_monodomain_create(&a->m, d);
    if (rc) { free(a); return rc; }
    mb_monodomain *m = a->m;
    a->nsteps = nsteps;
    a->every = checkpoint_every;
    a->ns = n_sensors;
    a->sample_every = sample_every;
    a->nsamples = nsteps / sample_every;
    a->nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
    a->snap = mb_tissue_snapshot_bytes(m);
    a->alpha = m->st.alpha;
    a->mx = (d->dy * d->dz) / d->dx;
    a->my = (d->dx * d->dz) / d->dy;
    a->mz = (d->dx * d->dy) / d->dz;
    const size_t ld = m->ode.ld, nb = (size_t)n * sizeof(double), rows = (size_t)MB_NEQ_TT2006 * ld * sizeof(double);
    cudaError_t e = cudaSuccess;
#define AALLOC(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    AALLOC(a->d_sensors, (size_t)n_sensors * sizeof(int64_t));
    AALLOC(a->d_ckpt, a->snap * (size_t)(a->nseg + 1));
    AALLOC(a->d_seg, a->snap * (size_t)(checkpoint_every + 1));
    AALLOC(a->d_traces, (size_t)(a->nsamples + 1) * n_sensors * sizeof(double));
    AALLOC(a->d_g, (size_t)(a->nsamples + 1) * n_sensors * sizeof(double));
    AALLOC(a->d_lam, nb);
    AALLOC(a->d_lam2, nb);
    AALLOC(a->d_w, nb);
    AALLOC(a->d_mu, rows);
    AALLOC(a->d_mu2, rows);
    AALLOC(a->d_gsig, nb);
    AALLOC(a->d_gth, ld * sizeof(double));
    AALLOC(a->d_sigma, nb);
    AALLOC(a->d_actrl, sizeof(mb_ctrl));
#undef AALLOC
    if (e == cudaSuccess)
        e = cudaMemcpy(a->d_sensors, sensor_cells, (size_t)n_sensors * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(a->d_sigma, d->sigma_cell, nb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        mb_adjoint_destroy(a);
        return AERR(MB_ERR_NOMEM, cudaGetErrorString(e));
    }
    /* the initial state, restored by every forward run */
    rc = mb_tissue_snapshot(m, a->d_ckpt + a->snap * (size_t)a->nseg, 0);
    if (!rc && cudaStreamSynchronize(m->stream) != cudaSuccess) rc = AERR(MB_ERR_CUDA, "snapshot");
    if (rc) { mb_adjoint_destroy(a); return rc; }
    *out = a;
    return MB_OK;
}

int mb_adjoint_forward(mb_adjoint *a, const double *sigma_cell, const double *scale, double *traces) {
    if (!a) return AERR(MB_ERR_ARG, "null");
    mb_monodomain *m = a->m;
    int rc;
    if (sigma_cell) {
        if ((rc = mb_tissue_set_sigma(m, sigma_cell))) return rc;
        ACK(cudaMemcpy(a->d_sigma, sigma_cell, (size_t)m->n * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (scale && (rc = mb_tissue_set_scale(m, scale))) return rc;
    if ((rc = mb_tissue_snapshot(m, a->d_ckpt + a->snap * (size_t)a->nseg, 1))) return rc;
    int sample = 0;
    for (int step = 0; step < a->nsteps; ++step) {
        if (step % a->every == 0 && (rc = mb_tissue_snapshot(m, a->d_ckpt + a->snap * (size_t)(step / a->every), 0)))
            return rc;
        if ((rc = mb_monodomain_step(m, 1))) return rc;
        if ((step + 1) % a->sample_every == 0 && sample < a->nsamples) {
            AKK(mbk_adj_gather(m->d_v, a->d_sensors, a->ns, a->d_traces + (size_t)sample * a->ns, m->stream));
            ++sample;
        }
    }
    if ((rc = mb_monodomain_sync(m))) return rc;
    if (traces)
        ACK(cudaMemcpy(traces, a->d_traces, (size_t)a->nsamples * a->ns * sizeof(double), cudaMemcpyDeviceToHost));
    a->have_forward = 1;
    return MB_OK;
}

int mb_adjoint_backward(mb_adjoint *a, const double *dtraces, double *grad_sigma, double *grad_scale_gkr) {
    if (!a || !dtraces) return AERR(MB_ERR_ARG, "null");
    if (!a->have_forward) return AERR(MB_ERR_STATE, "mb_adjoint_backward before mb_adjoint_forward");
    mb_monodomain *m = a->m;
    cudaStream_t s = m->stream;
    const int64_t n = m->n;
    const size_t ld = m->ode.ld, nb = (size_t)n * sizeof(double), rows = (size_t)MB_NEQ_TT2006 * ld * sizeof(double);
    int rc;
    ACK(cudaMemcpy(a->d_g, dtraces, (size_t)a->nsamples * a->ns * sizeof(double), cudaMemcpyHostToDevice));
    ACK(cudaMemsetAsync(a->d_lam, 0, nb, s));
    ACK(cudaMemsetAsync(a->d_w, 0, nb, s));
    ACK(cudaMemsetAsync(a->d_mu, 0, rows, s));
    ACK(cudaMemsetAsync(a->d_gsig, 0, nb, s));
    ACK(cudaMemsetAsync(a->d_gth, 0, ld * sizeof(double), s));
    /* control block of the transposed solves: the tissue's, with its own
     * tolerance (relative to lambda) and iteration limit */
    {
        mb_ctrl c;
        ACK(cudaMemcpy(&c, m->d_ctrl, sizeof c, cudaMemcpyDeviceToHost));
        c.max_its = 1000;
        c.use_precond = 1;
        ACK(cudaMemcpy(a->d_actrl, &c, sizeof c, cudaMemcpyHostToDevice));
    }
    mb_pcg_dev q = m->pcg;
    /* the z-march kernel's tensor maps address the tissue's own vectors (the
     * per-cell operator of the adjoint never selects it) */
    if (q.form == MB_PCG_ZMARCH) return AERR(MB_ERR_UNSUPPORTED, "the adjoint's transposed solve on the z-march CG");
    q.ctrl = a->d_actrl;
    q.x = a->d_w;
    q.b = a->d_lam;
    q.vstar = NULL;
    mb_ode_dev o = m->ode;

    for (int seg = a->nseg - 1; seg >= 0; --seg) {
        const int n0 = seg * a->every, n1 = (n0 + a->every < a->nsteps) ? n0 + a->every : a->nsteps;
        /* recompute the segment: snapshot k holds the state before step n0 + k */
        if ((rc = mb_tissue_snapshot(m, a->d_ckpt + a->snap * (size_t)seg, 1))) return rc;
        for (int k = 0; k <= n1 - n0; ++k) {
            if ((rc = mb_tissue_snapshot(m, a->d_seg + a->snap * (size_t)k, 0))) return rc;
            if (k < n1 - n0 && (rc = mb_monodomain_step(m, 1))) return rc;
        }
        for (int step = n1 - 1; step >= n0; --step) {
            const int k = step - n0;
            /* sampled gradient of v_{step+1} */
            if ((step + 1) % a->sample_every == 0) {
                const int sample = (step + 1) / a->sample_every - 1;
                if (sample < a->nsamples)
                    AKK(mbk_adj_scatter(a->d_lam, a->d_sensors, a->ns, a->d_g + (size_t)sample * a->ns, s));
            }
            double *v1, *v0, *sv0;
            mb_ctrl *c0;
            void *snap0 = a->d_seg + a->snap * (size_t)k;
            mb_tissue_snapshot_parts(m, a->d_seg + a->snap * (size_t)(k + 1), &v1, NULL, NULL);
            mb_tissue_snapshot_parts(m, snap0, &v0, &sv0, &c0);
            /* A w = lambda_{step+1} (warm start from the previous w) */
            AKK(mbk_adj_tol(a->d_lam, n, 1e-24, a->d_actrl, s));
            AKK(mbk_fcg_launch(&q, s));
            /* conductivity gradient through A(sigma) at v_{step+1} */
            AKK(mbk_adj_face_grad(&m->st, a->d_sigma, a->d_w, v1, a->mx, a->my, a->mz, a->d_gsig, s));
            /* through the Rush-Larsen step at (v_step, s_step) */
            ACK(cudaMemsetAsync(a->d_lam2, 0, nb, s));
            if (m->desc.precision == MB_PREC_MIXED)
                AKK(mbk_adj_tt2006_mixed(&o, c0, v0, sv0, mb_tissue_snapshot_sv32(m, snap0), a->d_w, a->alpha,
                                         a->d_mu, a->d_mu2, a->d_lam2, a->d_gth, s));
            else
                AKK(mbk_adj_tt2006(&o, c0, v0, sv0, a->d_w, a->alpha, a->d_mu, a->d_mu2, a->d_lam2, a->d_gth, s));
            double *t = a->d_lam; a->d_lam = a->d_lam2; a->d_lam2 = t;
            t = a->d_mu; a->d_mu = a->d_mu2; a->d_mu2 = t;
            q.b = a->d_lam;
        }
    }
    ACK(cudaStreamSynchronize(s));
    {
        int st = 0;
        ACK(cudaMemcpy(&st, m->d_status, sizeof st, cudaMemcpyDeviceToHost));
        if (st) return AERR(MB_ERR_CUDA, "CG grid barrier timed out in the adjoint");
    }
    if (grad_sigma) {
        ACK(cudaMemcpy(grad_sigma, a->d_gsig, nb, cudaMemcpyDeviceToHost));
        if (m->h_mask)
            for (int64_t g = 0; g < n; ++g)
                if (!m->h_mask[g]) grad_sigma[g] = 0.0;
    }
    if (grad_scale_gkr) {
        double *h = (double *)malloc(ld * sizeof(double));
        if (!h) return AERR(MB_ERR_NOMEM, "host memory");
        cudaError_t e = cudaMemcpy(h, a->d_gth, ld * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { free(h); return AERR(MB_ERR_CUDA, cudaGetErrorString(e)); }
        uint32_t t = 0;
        for (int64_t g = 0; g < n; ++g) {
            if (m->h_mask && !m->h_mask[g]) { grad_scale_gkr[g] = 0.0; continue; }
            grad_scale_gkr[g] = h[t++];
        }
        free(h);
    }
    /* the tissue holds the recomputed first segment's end; the next forward
     * run restores the initial state */
    return MB_OK;
}

/* The operator-split monodomain time loop on the CPU, FP64 -- TEST
 * INFRASTRUCTURE (oracle).  One orc_step is one iteration of
 * solve_monodomain's loop (src/monodomain/monodomain_solver.c:616-925,
 * without output, ECG and Purkinje):
 *
 *   cur_time > 0: sv[V] = cell->v                 (:660-661, :1012-1105)
 *   solve_all_volumes_odes: merged stimulus per cell, summed over the
 *     sub-steps whose time lies in [start, start + duration], then num_steps
 *     sub-steps of the cell model                  (ode_solver.c:183-248)
 *   update_monodomain_default: b = ALPHA * sv[V]   (update_monodomain.c:19-56)
 *   conjugate_gradient with x0 = cell->v           (linear_system_solver.c:47-183)
 *   NaN error stops the run                        (:746-754)
 *   cur_time += dt_pde                             (:907-908)
 *
 * The per-cell stimulus values follow stim_if_x_less_than, stim_x_y_limits and
 * stim_x_y_z_limits (stimuli.c:56-91,426-520) on cell centres
 * ((i + 1/2) dx, (j + 1/2) dy, (k + 1/2) dz), as set_cuboid_domain_mesh
 * places them (domain_helpers.c:19-73); initial conditions follow
 * set_initial_conditions_fvm (matrix_assembly.c:27-45) and the models'
 * set_model_initial_conditions_cpu.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

struct orc_sim {
    mb_monodomain_desc d;
    orc_csr A;
    int32_t n;            /* active cells (rows)                */
    int32_t *cells;       /* grid index of each row             */
    int neq;
    double *sv;           /* AoS state, neq per cell            */
    double *v;            /* cell->v, per row                   */
    double *b, *merged;
    double *stim_val;     /* MB_MAX_STIMS x n persistent values */
    double stim_start[MB_MAX_STIMS];
    uint8_t *celltype;    /* per row                            */
    double *scale;        /* 5 per row or NULL                  */
    double alpha;
    double cur_time;
    int num_steps;
    uint32_t last_its;
    double last_error;
};

int orc_loop_steps(double final_time, double dt) {
    double t = 0.0;
    int n = 0;
    while (t - final_time <= dt) {
        t += dt;
        n++;
    }
    return n;
}

static double stim_value(const mb_stim *st, int nx, int ny, int64_t g, double dx, double dy, double dz) {
    const int i = (int)(g % nx), j = (int)((g / nx) % ny), k = (int)(g / ((int64_t)nx * ny));
    const double cx = (i + 0.5) * dx, cy = (j + 0.5) * dy, cz = (k + 0.5) * dz;
    int on = 0;
    switch (st->kind) {
    case MB_STIM_X_LESS_THAN: on = cx < st->x_limit; break;
    case MB_STIM_X_Y_LIMITS:
        on = cx >= st->min[0] && cx <= st->max[0] && cy >= st->min[1] && cy <= st->max[1];
        break;
    case MB_STIM_X_Y_Z_LIMITS:
        on = cx >= st->min[0] && cx <= st->max[0] && cy >= st->min[1] && cy <= st->max[1] && cz >= st->min[2] &&
             cz <= st->max[2];
        break;
    case MB_STIM_CELL_MASK: on = st->cell_mask && st->cell_mask[g]; break;
    default: break;
    }
    return on ? st->current : 0.0;
}

void orc_stim_values(const mb_monodomain_desc *d, const int32_t *cells, int32_t n, double *out) {
    for (int k = 0; k < d->num_stims; ++k)
        for (int32_t c = 0; c < n; ++c)
            out[(size_t)k * n + c] = stim_value(&d->stims[k], d->nx, d->ny, cells[c], d->dx, d->dy, d->dz);
}

int orc_create(orc_sim **out, const mb_monodomain_desc *d) {
    if (!out || !d || d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || d->num_stims < 0 || d->num_stims > MB_MAX_STIMS)
        return MB_ERR_ARG;
    orc_sim *s = calloc(1, sizeof(orc_sim));
    if (!s) return MB_ERR_NOMEM;
    s->d = *d;
    const int64_t ng = (int64_t)d->nx * d->ny * d->nz;
    s->cells = malloc(sizeof(int32_t) * ng);
    int rc = s->cells ? orc_assemble(d, &s->A, s->cells) : MB_ERR_NOMEM;
    if (rc) { free(s->cells); free(s); return rc; }
    const int32_t n = s->n = s->A.n;
    s->neq = d->model == MB_MODEL_TT2006 ? ORC_TT_NEQ : ORC_TOR_NEQ;
    s->sv = malloc(sizeof(double) * (size_t)n * s->neq);
    s->v = malloc(sizeof(double) * (size_t)n);
    s->b = malloc(sizeof(double) * (size_t)n);
    s->merged = malloc(sizeof(double) * (size_t)n);
    s->stim_val = calloc((size_t)MB_MAX_STIMS * n + 1, sizeof(double));
    s->celltype = calloc((size_t)n + 1, 1);
    if (!s->sv || !s->v || !s->b || !s->merged || !s->stim_val || !s->celltype) { orc_destroy(s); return MB_ERR_NOMEM; }
    if (d->current_scale) {
        s->scale = malloc(sizeof(double) * (size_t)n * MB_NUM_SCALES);
        if (!s->scale) { orc_destroy(s); return MB_ERR_NOMEM; }
        for (int32_t c = 0; c < n; ++c)
            for (int q = 0; q < MB_NUM_SCALES; ++q)  /* the device keeps the scalings as float */
                s->scale[(size_t)c * MB_NUM_SCALES + q] = (double)(float)d->current_scale[q * ng + s->cells[c]];
    }
    s->alpha = (((d->beta * d->cm) / d->dt_pde) * (double)1.0e-8f) * (d->dx * d->dy * d->dz);
    s->num_steps = (int)(d->dt_pde / d->dt_ode);
    if (s->num_steps < 1) s->num_steps = 1;

    double v0;
    if (!isnan(d->initial_v)) v0 = d->initial_v;
    else v0 = d->model == MB_MODEL_TT2006 ? (double)-85.23f : -88.763800;
    for (int32_t c = 0; c < n; ++c) {
        double *y = s->sv + (size_t)c * s->neq;
        const int ct = d->celltype ? d->celltype[s->cells[c]] : 0;
        s->celltype[c] = (uint8_t)ct;
        if (d->initial_state) memcpy(y, d->initial_state, sizeof(double) * s->neq);
        else if (d->model == MB_MODEL_TT2006) orc_tt2006_initial_state(y);
        else orc_torord_initial_state(ct, y);
        s->v[c] = v0;
    }
    for (int k = 0; k < d->num_stims; ++k) {
        s->stim_start[k] = d->stims[k].start;
        for (int32_t c = 0; c < n; ++c)
            s->stim_val[(size_t)k * n + c] = stim_value(&d->stims[k], d->nx, d->ny, s->cells[c], d->dx, d->dy, d->dz);
    }
    *out = s;
    return MB_OK;
}

int orc_step(orc_sim *s, int nsteps) {
    const mb_monodomain_desc *d = &s->d;
    const int32_t n = s->n;
    const int neq = s->neq;
    const double dt = d->dt_ode;
    for (int step = 0; step < nsteps; ++step) {
        const double cur_time = s->cur_time;
        if (cur_time > 0.0) {
            for (int32_t c = 0; c < n; ++c) s->sv[(size_t)c * neq] = s->v[c];
        }
        /* merged stimulus (ode_solver.c:193-239) */
        for (int32_t c = 0; c < n; ++c) s->merged[c] = 0.0;
        for (int k = 0; k < d->num_stims; ++k) {
            const double start = s->stim_start[k], dur = d->stims[k].duration, period = d->stims[k].period;
            double time = cur_time;
            for (int j = 0; j < s->num_steps; ++j) {
                if (time >= start && time <= start + dur)
                    for (int32_t c = 0; c < n; ++c) s->merged[c] += s->stim_val[(size_t)k * n + c];
                time += dt;
            }
            if (period > 0.0 && time >= start + period) s->stim_start[k] = start + period;
        }
        /* the cell model (solve_model_odes_cpu) */
#pragma omp parallel for
        for (int32_t c = 0; c < n; ++c) {
            double *y = s->sv + (size_t)c * neq;
            const double *sc = s->scale ? s->scale + (size_t)c * MB_NUM_SCALES : NULL;
            for (int j = 0; j < s->num_steps; ++j) {
                if (d->model == MB_MODEL_TT2006) orc_tt2006_step(y, s->merged[c], dt, sc);
                else orc_torord_step(y, s->merged[c], dt, s->celltype[c], d->rl_rule, sc);
            }
        }
        /* update_monodomain_default */
        for (int32_t c = 0; c < n; ++c) s->b[c] = s->sv[(size_t)c * neq] * s->alpha;
        /* conjugate_gradient, x0 = cell->v */
        orc_pcg(&s->A, s->b, s->v, d->cg_tolerance, d->cg_max_iterations, d->use_preconditioner, &s->last_its,
                &s->last_error);
        if (isnan(s->last_error)) return MB_ERR_NAN;
        s->cur_time = cur_time + d->dt_pde;
    }
    return MB_OK;
}

void orc_get_v(const orc_sim *s, double *v_grid) {
    const int64_t ng = (int64_t)s->d.nx * s->d.ny * s->d.nz;
    for (int64_t g = 0; g < ng; ++g) v_grid[g] = NAN;
    for (int32_t c = 0; c < s->n; ++c) v_grid[s->cells[c]] = s->v[c];
}

void orc_get_state(const orc_sim *s, int var, double *out) {
    for (int32_t c = 0; c < s->n; ++c) out[c] = s->sv[(size_t)c * s->neq + var];
}

void orc_last_cg(const orc_sim *s, uint32_t *its, double *error) {
    if (its) *its = s->last_its;
    if (error) *error = s->last_error;
}

double orc_time(const orc_sim *s) { return s->cur_time; }
int32_t orc_active_cells(const orc_sim *s) { return s->n; }

void orc_destroy(orc_sim *s) {
    if (!s) return;
    orc_csr_free(&s->A);
    free(s->cells); free(s->sv); free(s->v); free(s->b); free(s->merged);
    free(s->stim_val); free(s->celltype); free(s->scale);
    free(s);
}

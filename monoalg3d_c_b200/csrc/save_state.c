/* Checkpoints in the reference's own layout: the three files that
 * save_simulation_state writes and restore_simulation_state reads
 * (src/save_state_library/save_state.c:16-150,
 *  src/restore_state_library/restore_state.c:38-230):
 *
 *   grid_checkpoint.dat               cube and mesh side lengths, number of
 *                                     cells (every leaf of the reference's
 *                                     octree, inactive ones included) and of
 *                                     active cells; then per leaf, in the
 *                                     octree's list order: centre, V, six
 *                                     fluxes, b, can_change, active, size of
 *                                     the extra mesh data (none here);
 *   monodomain_solver_checkpoint.dat  struct monodomain_solver, struct time_info;
 *   ode_solver_checkpoint.dat         adaptive, max_dt, min_dt, rel_tol,
 *                                     abs_tol, num_cells_to_solve, (no
 *                                     cells_to_solve), gpu, gpu_id, pitch,
 *                                     original_num_cells, then the state
 *                                     vector: cell after cell (CPU build) or
 *                                     state row after state row (GPU build).
 *
 * The reference restores the grid records by cell centre, but reads the state
 * vector as it lies, so its rows must be in the reference's numbering of the
 * active cells: the order of the leaves of its octree, which its cell
 * refinement walks along a Hilbert curve (cell_refinement.c:510-1160,
 * order_grid_cells in grid.c:245-263).  For a cuboid of nx x ny x nz cells the
 * octree is a cube of 2^L cells (L = ceil(log2(max(nx, ny, nz))), at least 1)
 * refined to single cells wherever it meets the cuboid; a node wholly outside
 * the cuboid stays one inactive leaf.  Every node visits its eight children in
 * the order its curve shape gives, and hands each child a shape: the table
 * below (octant code 4 x + 2 y + z of each child in visiting order, and the
 * child's shape), read from the reference's own grid builder by
 * oracle/ref/hilbert_probe.c and checked against it on several cuboids.
 * Removed cells of a mask stay single-cell leaves with active = false, as the
 * reference's fibrosis marks them after building the cuboid.
 */
#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <cuda_runtime_api.h>

#include <stdarg.h>

#include "mb_tissue.h"

static int fail(int code, const char *fmt, ...) {
    char msg[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    return mb_internal_error(code, msg);
}

static const uint8_t HILBERT_CHILD[12][8] = {
    {7, 3, 1, 5, 4, 0, 2, 6}, {7, 6, 4, 5, 1, 0, 2, 3}, {7, 3, 2, 6, 4, 0, 1, 5}, {1, 5, 7, 3, 2, 6, 4, 0},
    {4, 0, 1, 5, 7, 3, 2, 6}, {2, 3, 1, 0, 4, 5, 7, 6}, {2, 6, 7, 3, 1, 5, 4, 0}, {4, 0, 2, 6, 7, 3, 1, 5},
    {1, 3, 2, 0, 4, 6, 7, 5}, {4, 5, 7, 6, 2, 3, 1, 0}, {1, 0, 4, 5, 7, 6, 2, 3}, {2, 6, 4, 0, 1, 5, 7, 3}};
static const uint8_t HILBERT_NEXT[12][8] = {
    {1, 2, 2, 3, 3, 4, 4, 5},     {0, 2, 2, 9, 9, 10, 10, 11}, {1, 0, 0, 6, 6, 7, 7, 8},  {8, 10, 10, 0, 0, 6, 6, 9},
    {9, 7, 7, 10, 10, 0, 0, 5},   {11, 6, 6, 8, 8, 4, 4, 0},   {5, 11, 11, 2, 2, 3, 3, 9}, {9, 4, 4, 11, 11, 2, 2, 8},
    {10, 3, 3, 5, 5, 7, 7, 2},    {7, 4, 4, 1, 1, 6, 6, 3},    {3, 8, 8, 4, 4, 1, 1, 11},  {5, 6, 6, 7, 7, 10, 10, 1}};

/* ---- the octree walk ------------------------------------------------------ */

typedef struct {
    int nx, ny, nz, L;
    /* per leaf: x0, y0, z0 (cells), side (cells), inside (a single cell of the cuboid) */
    void (*leaf)(void *ctx, int x0, int y0, int z0, int side, int inside);
    void *ctx;
} walk_t;

static void walk(const walk_t *w, int x0, int y0, int z0, int level, int shape) {
    const int side = 1 << (w->L - level);
    const int outside = x0 >= w->nx || y0 >= w->ny || z0 >= w->nz;
    if (level >= 1 && outside) {
        w->leaf(w->ctx, x0, y0, z0, side, 0);
        return;
    }
    if (level == w->L) {
        w->leaf(w->ctx, x0, y0, z0, 1, 1);
        return;
    }
    const int h = side >> 1;
    for (int q = 0; q < 8; ++q) {
        const int o = HILBERT_CHILD[shape][q];
        walk(w, x0 + ((o >> 2) & 1) * h, y0 + ((o >> 1) & 1) * h, z0 + (o & 1) * h, level + 1, HILBERT_NEXT[shape][q]);
    }
}

static int levels_of(int nx, int ny, int nz) {
    int m = nx > ny ? nx : ny;
    if (nz > m) m = nz;
    int L = 1;
    while ((1 << L) < m) ++L;
    return L;
}

typedef struct {
    const uint8_t *active;
    int nx, ny;
    int64_t *order;
    int64_t n_active, n_leaves;
} order_ctx;

static void order_leaf(void *c, int x0, int y0, int z0, int side, int inside) {
    order_ctx *o = (order_ctx *)c;
    (void)side;
    o->n_leaves++;
    if (!inside) return;
    const int64_t g = (int64_t)x0 + (int64_t)o->nx * ((int64_t)y0 + (int64_t)o->ny * z0);
    if (o->active && !o->active[g]) return;
    if (o->order) o->order[o->n_active] = g;
    o->n_active++;
}

int mb_reference_cell_order(int nx, int ny, int nz, const uint8_t *active, int64_t *order, int64_t *n_active,
                            int64_t *number_of_cells) {
    if (nx < 1 || ny < 1 || nz < 1) return fail(MB_ERR_ARG, "grid sizes must be positive");
    order_ctx o = {active, nx, ny, order, 0, 0};
    walk_t w = {nx, ny, nz, levels_of(nx, ny, nz), order_leaf, &o};
    walk(&w, 0, 0, 0, 0, 0);
    if (n_active) *n_active = o.n_active;
    if (number_of_cells) *number_of_cells = o.n_leaves;
    return MB_OK;
}

/* ---- file layouts ------------------------------------------------------------ */

/* struct monodomain_solver and struct time_info of the reference
 * (monodomain_solver.h:16-36, common_types.h:78-83), member for member: the
 * reference writes and reads them with fwrite / fread of the whole struct. */
typedef struct {
    int num_threads;
    double final_time;
    double beta, cm;
    int refine_each;
    int derefine_each;
    double refinement_bound;
    double derefinement_bound;
    double start_adapting_at;
    bool abort_on_no_activity;
    double only_abort_after_dt;
    double dt;
} ref_monodomain_solver;

typedef struct {
    double current_t, final_t, dt;
    int iteration;
} ref_time_info;

typedef struct {
    FILE *f;
    const double *v, *vstar;
    const uint8_t *mask;
    double alpha, dx, dy, dz;
    int nx, ny;
    int ok;
} write_ctx;

static void put(write_ctx *w, const void *p, size_t n) {
    if (w->ok && fwrite(p, 1, n, w->f) != n) w->ok = 0;
}

static void write_leaf(void *c, int x0, int y0, int z0, int side, int inside) {
    write_ctx *w = (write_ctx *)c;
    const double h = 0.5 * side;
    const double center[3] = {(x0 + h) * w->dx, (y0 + h) * w->dy, (z0 + h) * w->dz};
    double v = 0.0, b = 0.0;
    bool active = false;
    if (inside) {
        const int64_t g = (int64_t)x0 + (int64_t)w->nx * ((int64_t)y0 + (int64_t)w->ny * z0);
        active = !w->mask || w->mask[g];
        if (active) {
            v = w->v[g];
            b = w->alpha * w->vstar[g];
        }
    }
    const double flux[6] = {0, 0, 0, 0, 0, 0};
    const bool can_change = true;
    const size_t extra = 0;
    put(w, center, sizeof center);
    put(w, &v, sizeof v);
    put(w, flux, sizeof flux);
    put(w, &b, sizeof b);
    put(w, &can_change, sizeof can_change);
    put(w, &active, sizeof active);
    put(w, &extra, sizeof extra);
}

static FILE *open_in(const char *dir, const char *name, const char *mode) {
    char path[4096];
    snprintf(path, sizeof path, "%s/%s", dir, name);
    return fopen(path, mode);
}

/* Host copies of V, V* and the dense state (neq x n_active, compact order). */
static int fetch(mb_monodomain *m, double **v, double **vstar, double **state, mb_ctrl *ctrl) {
    const size_t n = (size_t)m->n, na = m->n_active;
    *v = (double *)malloc(n * sizeof(double));
    *vstar = (double *)malloc(n * sizeof(double));
    *state = (double *)malloc((size_t)m->neq * na * sizeof(double));
    if (!*v || !*vstar || !*state) return fail(MB_ERR_NOMEM, "host memory");
    double *d = NULL;
    cudaError_t e = cudaStreamSynchronize(m->stream);
    if (e == cudaSuccess) e = cudaMalloc((void **)&d, (size_t)m->neq * na * sizeof(double));
    /* state row 0 holds V* (the ODE's output of the last step), as the
     * reference's sv does at a step boundary */
    if (e == cudaSuccess) e = (cudaError_t)mbk_ode_gather(&m->ode, m->d_vstar, d, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(*state, d, (size_t)m->neq * na * sizeof(double), cudaMemcpyDeviceToHost,
                                              m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(*v, m->d_v, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(*vstar, m->d_vstar, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctrl, m->d_ctrl, sizeof *ctrl, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(d);
    return e == cudaSuccess ? MB_OK : fail(MB_ERR_CUDA, "%s", cudaGetErrorString(e));
}

/* Row pitch cudaMallocPitch gives a state row of n doubles on this device
 * (the GPU build's sv, ten_tusscher_2006_RS_GPU.cu:20). */
static size_t pitch_of(size_t n) {
    void *p = NULL;
    size_t pitch = n * sizeof(double);
    if (cudaMallocPitch(&p, &pitch, n * sizeof(double), 1) == cudaSuccess) cudaFree(p);
    else cudaGetLastError();
    return pitch;
}

int mb_monodomain_save_state(mb_monodomain *m, const char *dir, int gpu_layout) {
    if (!m || !dir) return fail(MB_ERR_ARG, "null");
    const mb_monodomain_desc *d = &m->desc;
    double *v = NULL, *vstar = NULL, *state = NULL;
    int64_t *order = NULL;
    mb_ctrl c;
    int rc = fetch(m, &v, &vstar, &state, &c);
    if (rc) goto done;
    order = (int64_t *)malloc((size_t)m->n_active * sizeof(int64_t));
    int64_t na = 0, leaves = 0;
    if (!order) { rc = fail(MB_ERR_NOMEM, "host memory"); goto done; }
    rc = mb_reference_cell_order(d->nx, d->ny, d->nz, m->h_mask, order, &na, &leaves);
    if (rc) goto done;
    if (na != (int64_t)m->n_active || leaves > 0xffffffffLL) {
        rc = fail(MB_ERR_STATE, "cell numbering does not match the tissue");
        goto done;
    }
    /* grid */
    {
        FILE *f = open_in(dir, "grid_checkpoint.dat", "wb");
        if (!f) { rc = fail(MB_ERR_ARG, "cannot write grid_checkpoint.dat in %s", dir); goto done; }
        const int L = levels_of(d->nx, d->ny, d->nz);
        const double cube[3] = {d->dx * (1 << L), d->dy * (1 << L), d->dz * (1 << L)};
        const double mesh[3] = {d->dx * d->nx, d->dy * d->ny, d->dz * d->nz};
        const uint32_t ncells = (uint32_t)leaves, nact = (uint32_t)na;
        write_ctx w = {f, v, vstar, m->h_mask, m->st.alpha, d->dx, d->dy, d->dz, d->nx, d->ny, 1};
        put(&w, cube, sizeof cube);
        put(&w, mesh, sizeof mesh);
        put(&w, &ncells, sizeof ncells);
        put(&w, &nact, sizeof nact);
        walk_t wk = {d->nx, d->ny, d->nz, L, write_leaf, &w};
        walk(&wk, 0, 0, 0, 0, 0);
        if (fclose(f) != 0 || !w.ok) { rc = fail(MB_ERR_ARG, "writing grid_checkpoint.dat failed"); goto done; }
    }
    /* monodomain solver and clock */
    {
        FILE *f = open_in(dir, "monodomain_solver_checkpoint.dat", "wb");
        if (!f) { rc = fail(MB_ERR_ARG, "cannot write the solver checkpoint in %s", dir); goto done; }
        ref_monodomain_solver s;
        memset(&s, 0, sizeof s);
        long cpus = sysconf(_SC_NPROCESSORS_ONLN);
        s.num_threads = cpus > 0 ? (int)cpus : 1;
        s.final_time = c.cur_time;
        s.beta = d->beta;
        s.cm = d->cm;
        /* the adaptivity fields at the reference's option defaults
         * (config_parser.c:288-340, monodomain_solver.c:1310-1331) */
        s.refine_each = 1;
        s.derefine_each = 1;
        s.refinement_bound = 0.11;
        s.derefinement_bound = 0.1;
        s.start_adapting_at = 1.0;
        s.dt = d->dt_pde;
        ref_time_info t = {c.cur_time, c.cur_time, d->dt_pde, (int)c.count};
        const int ok = fwrite(&s, sizeof s, 1, f) == 1 && fwrite(&t, sizeof t, 1, f) == 1;
        if (fclose(f) != 0 || !ok) { rc = fail(MB_ERR_ARG, "writing the solver checkpoint failed"); goto done; }
    }
    /* ODE state, rows in the reference's cell numbering */
    {
        FILE *f = open_in(dir, "ode_solver_checkpoint.dat", "wb");
        if (!f) { rc = fail(MB_ERR_ARG, "cannot write the ODE checkpoint in %s", dir); goto done; }
        const size_t ncomp = m->n_active;
        /* compact index of every grid cell */
        int64_t *comp = (int64_t *)malloc((size_t)m->n * sizeof(int64_t));
        if (!comp) { fclose(f); rc = fail(MB_ERR_NOMEM, "host memory"); goto done; }
        for (int64_t g = 0, t = 0; g < m->n; ++g) comp[g] = (!m->h_mask || m->h_mask[g]) ? t++ : -1;
        const bool adaptive = false, read_cells = false, gpu = gpu_layout != 0;
        const double max_dt = d->dt_pde, min_dt = d->dt_ode, rel_tol = 1e-5, abs_tol = 1e-5;
        const size_t ntosolve = ncomp;
        const int gpu_id = 0;
        const size_t pitch = gpu ? pitch_of(ncomp) : 0;
        const uint32_t orig = (uint32_t)ncomp;
        int ok = fwrite(&adaptive, sizeof adaptive, 1, f) == 1 && fwrite(&max_dt, sizeof max_dt, 1, f) == 1 &&
                 fwrite(&min_dt, sizeof min_dt, 1, f) == 1 && fwrite(&rel_tol, sizeof rel_tol, 1, f) == 1 &&
                 fwrite(&abs_tol, sizeof abs_tol, 1, f) == 1 && fwrite(&ntosolve, sizeof ntosolve, 1, f) == 1 &&
                 fwrite(&read_cells, sizeof read_cells, 1, f) == 1 && fwrite(&gpu, sizeof gpu, 1, f) == 1 &&
                 fwrite(&gpu_id, sizeof gpu_id, 1, f) == 1 && fwrite(&pitch, sizeof pitch, 1, f) == 1 &&
                 fwrite(&orig, sizeof orig, 1, f) == 1;
        double *row = (double *)malloc((gpu ? ncomp : (size_t)m->neq) * sizeof(double));
        if (!row) ok = 0;
        if (gpu) {
            for (int s = 0; s < m->neq && ok; ++s) {
                for (size_t r = 0; r < ncomp; ++r) row[r] = state[(size_t)s * ncomp + comp[order[r]]];
                ok = fwrite(row, sizeof(double), ncomp, f) == ncomp;
            }
        } else {
            for (size_t r = 0; r < ncomp && ok; ++r) {
                for (int s = 0; s < m->neq; ++s) row[s] = state[(size_t)s * ncomp + comp[order[r]]];
                ok = fwrite(row, sizeof(double), (size_t)m->neq, f) == (size_t)m->neq;
            }
        }
        free(row);
        free(comp);
        if (fclose(f) != 0 || !ok) { rc = fail(MB_ERR_ARG, "writing the ODE checkpoint failed"); goto done; }
    }
done:
    free(v); free(vstar); free(state); free(order);
    return rc;
}

static int get(FILE *f, void *p, size_t n) {
    return fread(p, 1, n, f) == n;
}

int mb_monodomain_restore_state(mb_monodomain *m, const char *dir) {
    if (!m || !dir) return fail(MB_ERR_ARG, "null");
    const mb_monodomain_desc *d = &m->desc;
    double *v = NULL, *vstar = NULL, *state = NULL;
    int64_t *rank_to_grid = NULL, *comp = NULL;
    FILE *f = NULL;
    mb_ctrl c;
    int rc = fetch(m, &v, &vstar, &state, &c);
    if (rc) goto done;
    const size_t na = m->n_active;
    rank_to_grid = (int64_t *)malloc(na * sizeof(int64_t));
    comp = (int64_t *)malloc((size_t)m->n * sizeof(int64_t));
    if (!rank_to_grid || !comp) { rc = fail(MB_ERR_NOMEM, "host memory"); goto done; }
    for (int64_t g = 0, t = 0; g < m->n; ++g) comp[g] = (!m->h_mask || m->h_mask[g]) ? t++ : -1;
    /* grid: V by cell centre; the active records in file order are the
     * state vector's rows */
    f = open_in(dir, "grid_checkpoint.dat", "rb");
    if (!f) { rc = fail(MB_ERR_ARG, "cannot read grid_checkpoint.dat in %s", dir); goto done; }
    {
        double cube[3], mesh[3];
        uint32_t ncells, nact;
        if (!get(f, cube, sizeof cube) || !get(f, mesh, sizeof mesh) || !get(f, &ncells, 4) || !get(f, &nact, 4)) {
            rc = fail(MB_ERR_ARG, "grid_checkpoint.dat is truncated");
            goto done;
        }
        if (fabs(mesh[0] - d->nx * d->dx) > 1e-6 * mesh[0] || fabs(mesh[1] - d->ny * d->dy) > 1e-6 * mesh[1] ||
            fabs(mesh[2] - d->nz * d->dz) > 1e-6 * mesh[2] || nact != na) {
            rc = fail(MB_ERR_ARG, "the checkpoint's mesh (%g x %g x %g um, %u active cells) is not this "
                                   "tissue's", mesh[0], mesh[1], mesh[2], nact);
            goto done;
        }
        size_t r = 0;
        for (uint32_t q = 0; q < ncells; ++q) {
            double center[3], vv, flux[6], b;
            bool can_change, active;
            size_t extra;
            if (!get(f, center, sizeof center) || !get(f, &vv, 8) || !get(f, flux, sizeof flux) || !get(f, &b, 8) ||
                !get(f, &can_change, 1) || !get(f, &active, 1) || !get(f, &extra, sizeof extra)) {
                rc = fail(MB_ERR_ARG, "grid_checkpoint.dat is truncated");
                goto done;
            }
            if (extra && fseek(f, (long)extra, SEEK_CUR) != 0) {
                rc = fail(MB_ERR_ARG, "grid_checkpoint.dat is truncated");
                goto done;
            }
            if (!active) continue;
            const long i = lround(center[0] / d->dx - 0.5), j = lround(center[1] / d->dy - 0.5),
                       k = lround(center[2] / d->dz - 0.5);
            if (i < 0 || j < 0 || k < 0 || i >= d->nx || j >= d->ny || k >= d->nz || r >= na) {
                rc = fail(MB_ERR_ARG, "an active cell of the checkpoint lies outside this tissue");
                goto done;
            }
            const int64_t g = i + (int64_t)d->nx * (j + (int64_t)d->ny * k);
            if (comp[g] < 0) {
                rc = fail(MB_ERR_ARG, "the checkpoint's active cells are not this tissue's");
                goto done;
            }
            v[g] = vv;
            rank_to_grid[r++] = g;
        }
        if (r != na) { rc = fail(MB_ERR_ARG, "active cell count mismatch"); goto done; }
    }
    fclose(f);
    f = NULL;
    /* clock */
    f = open_in(dir, "monodomain_solver_checkpoint.dat", "rb");
    if (!f) { rc = fail(MB_ERR_ARG, "cannot read the solver checkpoint in %s", dir); goto done; }
    {
        ref_monodomain_solver s;
        ref_time_info t;
        if (!get(f, &s, sizeof s) || !get(f, &t, sizeof t)) {
            rc = fail(MB_ERR_ARG, "the solver checkpoint is truncated");
            goto done;
        }
        if (fabs(s.dt - d->dt_pde) > 1e-12 || fabs(s.beta - d->beta) > 1e-12 * fabs(d->beta) ||
            fabs(s.cm - d->cm) > 1e-12 * fabs(d->cm)) {
            rc = fail(MB_ERR_ARG, "the checkpoint's dt / beta / cm differ from this tissue's");
            goto done;
        }
        c.cur_time = t.current_t;
        c.count = t.iteration;
    }
    fclose(f);
    f = NULL;
    /* ODE state */
    f = open_in(dir, "ode_solver_checkpoint.dat", "rb");
    if (!f) { rc = fail(MB_ERR_ARG, "cannot read the ODE checkpoint in %s", dir); goto done; }
    {
        bool adaptive, read_cells, gpu;
        double max_dt, min_dt, rel_tol, abs_tol;
        size_t ntosolve, pitch;
        int gpu_id;
        uint32_t orig;
        if (!get(f, &adaptive, 1) || !get(f, &max_dt, 8) || !get(f, &min_dt, 8) || !get(f, &rel_tol, 8) ||
            !get(f, &abs_tol, 8) || !get(f, &ntosolve, sizeof ntosolve)) {
            rc = fail(MB_ERR_ARG, "the ODE checkpoint is truncated");
            goto done;
        }
        if (!get(f, &read_cells, 1)) { rc = fail(MB_ERR_ARG, "the ODE checkpoint is truncated"); goto done; }
        if (read_cells && fseek(f, (long)(ntosolve * sizeof(uint32_t)), SEEK_CUR) != 0) {
            rc = fail(MB_ERR_ARG, "the ODE checkpoint is truncated");
            goto done;
        }
        if (!get(f, &gpu, 1) || !get(f, &gpu_id, sizeof gpu_id) || !get(f, &pitch, sizeof pitch) ||
            !get(f, &orig, 4)) {
            rc = fail(MB_ERR_ARG, "the ODE checkpoint is truncated");
            goto done;
        }
        if (adaptive || orig != na) {
            rc = fail(MB_ERR_ARG, "the ODE checkpoint is adaptive or holds %u cells, not %zu", orig, na);
            goto done;
        }
        double *buf = (double *)malloc((size_t)m->neq * na * sizeof(double));
        if (!buf) { rc = fail(MB_ERR_NOMEM, "host memory"); goto done; }
        if (fread(buf, sizeof(double), (size_t)m->neq * na, f) != (size_t)m->neq * na) {
            free(buf);
            rc = fail(MB_ERR_ARG, "the ODE checkpoint is truncated");
            goto done;
        }
        for (size_t r = 0; r < na; ++r) {
            const int64_t t = comp[rank_to_grid[r]];
            for (int s = 0; s < m->neq; ++s)
                state[(size_t)s * na + t] = gpu ? buf[(size_t)s * na + r] : buf[r * m->neq + s];
        }
        free(buf);
    }
    fclose(f);
    f = NULL;
    /* upload: the state rows (row 0, V* at a step boundary, into V*), V on
     * the grid, the clock */
    {
        double *dd = NULL;
        cudaError_t e = cudaMalloc((void **)&dd, (size_t)m->neq * na * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpyAsync(dd, state, (size_t)m->neq * na * sizeof(double),
                                                  cudaMemcpyHostToDevice, m->stream);
        if (e == cudaSuccess) e = (cudaError_t)mbk_ode_scatter(&m->ode, dd, m->d_vstar, m->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_v, v, (size_t)m->n * sizeof(double), cudaMemcpyHostToDevice,
                                                  m->stream);
        c.w_valid = 0;           /* V comes from the file: no stored A x for it */
        if (e == cudaSuccess) e = cudaMemcpyAsync(m->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice, m->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
        cudaFree(dd);
        if (e != cudaSuccess) rc = fail(MB_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
done:
    if (f) fclose(f);
    free(v); free(vstar); free(state); free(rank_to_grid); free(comp);
    return rc;
}

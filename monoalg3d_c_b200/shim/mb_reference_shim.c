/* Reference-host plugins: the cell-model library and linear-solver entry
 * points of MonoAlg3D's plugin interface, implemented on this library's GPU
 * kernels.  The unmodified MonoAlg3D binary loads them through its own
 * dlopen/dlsym path (ode_solver.c:74-128, config_common.c:20-80) when an
 * ini points [ode_solver] library_file and [linear_system_solver]
 * library_file at the built shim, and runs its own time loop
 * (monodomain_solver.c:616-925) with the ODE and CG work on the GPU.
 *
 * The shim follows the reference's CPU data flow, so the orchestrator and
 * the other plugins see what they expect:
 *   - set_model_initial_conditions_cpu allocates the host state vector sv
 *     (neq x cells, array of structures, freed by the driver with free()) and
 *     fills it with the model's initial state;
 *   - solve_model_odes_cpu takes V from sv[i * neq] (written there by the
 *     orchestrator, monodomain_solver.c:1051), integrates num_steps sub-steps
 *     on the GPU with the merged stimulus array, and writes V* back to
 *     sv[i * neq] for update_monodomain_default (update_monodomain.c:50); the
 *     other states stay on the device;
 *   - conjugate_gradient uploads the assembled matrix once (each cell's
 *     elements in their stored order, diagonal first), then per call copies
 *     b and V in, runs the Jacobi-PCG on the GPU (same recurrences and
 *     stopping rule as cpu_conjugate_gradient,
 *     linear_system_solver.c:47-183) and writes V back to the cells.
 *
 * The GPU build of the reference (COMPILE_CUDA, [ode_solver] use_gpu = yes)
 * resolves the GPU entry points instead (ode_solver.c:114-126) and keeps the
 * state on the device:
 *   - set_model_initial_conditions_gpu hands the host this library's own
 *     device state as ode_solver->sv (pitched FP64 rows, V in row 0, the
 *     layout of the reference's GPU models, ten_tusscher_2006_RS_GPU.cu:8-40)
 *     and returns its pitch;
 *   - solve_model_odes_gpu integrates in place: the host writes V into row 0
 *     before the call (update_ode_state_vector, monodomain_solver.c:1026-1045)
 *     and update_monodomain_default reads V* from row 0 after it
 *     (update_monodomain.c:31-52); nothing crosses to the host.
 *
 * ToRORd extra data (set_extra_data_mixed_torord_fkatp_epi_mid_endo and the
 * like, struct extra_data_for_torord, helper_functions.h:44-68): the cell
 * type of every cell (transmurality) selects its initial state and its
 * currents; the initial states must be the reference's default steady states
 * and every current multiplier 1 (the defaults of set_common_torord_data,
 * helper_functions.c:94-160) -- other values are reported and fatal.
 *
 * Compiled against the reference's headers (struct layouts and the plugin
 * signature macros) with CELL_MODEL_REAL_DOUBLE, as the reference's default
 * build; no reference function is called.  MB_SHIM_MODEL selects the cell
 * model this copy provides.  Not supported (reported and fatal, as the
 * reference's fatal paths are): adaptive meshes / cells_to_solve, the
 * adaptive ODE step and Purkinje systems. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ode_solver/ode_solver.h"
#include "config/linear_system_solver_config.h"
#include "extra_data_library/helper_functions.h"
#include "3dparty/stb_ds.h"

#include "monoalg3d_b200.h"

#ifndef MB_SHIM_MODEL
#error "MB_SHIM_MODEL must name the cell model (MB_MODEL_TT2006, MB_MODEL_TORORD_FKATP_MIXED or MB_MODEL_TORORD_FKATP_ENDO)"
#endif

static void shim_fail(const char *what) {
    fprintf(stderr, "monoalg3d_b200 shim: %s: %s\n", what, mb_last_error());
    exit(1);
}

static void shim_check(int rc, const char *what) {
    if (rc != MB_OK) shim_fail(what);
}

/* ---- cell-model library (ode_solver.h:33-47) ---------------------------- */

static mb_ode *g_ode;        /* created at the first solve, when dt and num_steps are final */
static double *g_vbuf;       /* V of every cell, contiguous (CPU-build entry points) */
static uint32_t g_ode_cells;
static uint8_t *g_celltype;  /* ToRORd cell type of every cell (extra data), or NULL */

/* The cell types of the ToRORd extra data, checked against what this library
 * models (see the header comment); NULL when there is none. */
static uint8_t *torord_celltypes(struct ode_solver *solver, uint32_t n) {
    if (MB_SHIM_MODEL != MB_MODEL_TORORD_FKATP_MIXED || !solver->ode_extra_data || solver->extra_data_size == 0)
        return NULL;
    const struct extra_data_for_torord *x = (const struct extra_data_for_torord *)solver->ode_extra_data;
    const real mult[] = {x->INa_Multiplier, x->ICaL_Multiplier, x->Ito_Multiplier, x->INaL_Multiplier,
                         x->IKr_Multiplier, x->IKs_Multiplier, x->IK1_Multiplier, x->IKb_Multiplier,
                         x->INaCa_Multiplier, x->INaK_Multiplier, x->INab_Multiplier, x->ICab_Multiplier,
                         x->IpCa_Multiplier, x->ICaCl_Multiplier, x->IClb_Multiplier, x->Jrel_Multiplier,
                         x->Jup_Multiplier};
    for (size_t k = 0; k < sizeof mult / sizeof mult[0]; ++k)
        if (mult[k] != 1.0) {
            fprintf(stderr, "monoalg3d_b200 shim: ToRORd current multipliers other than 1 are not supported\n");
            exit(1);
        }
    const real *ic[3] = {x->initial_ss_endo, x->initial_ss_mid, x->initial_ss_epi};
    double def[43];
    for (int t = 0; t < 3; ++t) {
        shim_check(mb_torord_initial_state(t, def), "default initial state");
        for (int q = 0; q < 43 && ic[t]; ++q)
            if (ic[t][q] != (real)def[q]) {
                fprintf(stderr, "monoalg3d_b200 shim: ToRORd initial states other than the default steady "
                                "states are not supported\n");
                exit(1);
            }
    }
    uint8_t *ct = (uint8_t *)malloc(n ? n : 1);
    if (!ct) {
        fprintf(stderr, "monoalg3d_b200 shim: out of host memory\n");
        exit(1);
    }
    for (uint32_t i = 0; i < n; ++i) {
        const real t = x->transmurality ? x->transmurality[i] : 0.0;
        ct[i] = t == 1.0 ? 1 : (t == 2.0 ? 2 : 0);     /* ENDO 0, MID 1, EPI 2 */
    }
    return ct;
}

GET_CELL_MODEL_DATA(init_cell_model_data) {
    int neq = 0;
    double v0 = 0.0;
    shim_check(mb_init_cell_model_data(MB_SHIM_MODEL, &neq, &v0), "init_cell_model_data");
    if (get_initial_v) cell_model->initial_v = (real)v0;
    if (get_neq) cell_model->number_of_ode_equations = neq;
}

SET_ODE_INITIAL_CONDITIONS_CPU(set_model_initial_conditions_cpu) {
    (void)ode_extra_config;
    if (solver->adaptive || solver->cells_to_solve) {
        fprintf(stderr, "monoalg3d_b200 shim: adaptive meshes are not supported\n");
        exit(1);
    }
    const uint32_t n = solver->original_num_cells;
    free(g_celltype);
    g_celltype = torord_celltypes(solver, n);
    const int neq = solver->model_data.number_of_ode_equations;
    solver->sv = (real *)malloc((size_t)n * neq * sizeof(real));
    double *soa = (double *)malloc((size_t)n * neq * sizeof(double));
    if (!solver->sv || !soa) {
        fprintf(stderr, "monoalg3d_b200 shim: out of host memory\n");
        exit(1);
    }
    /* the model's initial state, from a one-step object of the same size */
    mb_ode *tmp = NULL;
    size_t pitch = 0;
    shim_check(mb_ode_create(&tmp, MB_SHIM_MODEL, MB_PREC_FP64, MB_RL_REFERENCE_CPU, n, 1.0, 1), "mb_ode_create");
    shim_check(mb_set_model_initial_conditions_gpu(tmp, NULL, g_celltype, &pitch), "initial conditions");
    shim_check(mb_ode_get_state(tmp, soa), "initial state");
    mb_ode_destroy(tmp);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        for (int s = 0; s < neq; ++s) solver->sv[(size_t)i * neq + s] = soa[(size_t)s * n + i];
    free(soa);
    if (g_ode) {
        mb_ode_destroy(g_ode);
        g_ode = NULL;
    }
    free(g_vbuf);
    g_vbuf = NULL;
}

SOLVE_MODEL_ODES(solve_model_odes_cpu) {
    (void)ode_extra_config;
    const uint32_t n = (uint32_t)ode_solver->num_cells_to_solve;
    const int neq = ode_solver->model_data.number_of_ode_equations;
    if (!g_ode) {
        /* the whole state from sv, in this library's row layout */
        double *soa = (double *)malloc((size_t)n * neq * sizeof(double));
        if (!soa) {
            fprintf(stderr, "monoalg3d_b200 shim: out of host memory\n");
            exit(1);
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i)
            for (int s = 0; s < neq; ++s) soa[(size_t)s * n + i] = ode_solver->sv[(size_t)i * neq + s];
        shim_check(mb_ode_create(&g_ode, MB_SHIM_MODEL, MB_PREC_FP64, MB_RL_REFERENCE_CPU, n, ode_solver->min_dt,
                                 ode_solver->num_steps),
                   "mb_ode_create");
        size_t pitch = 0;
        shim_check(mb_set_model_initial_conditions_gpu(g_ode, NULL, g_celltype, &pitch), "cell types");
        shim_check(mb_ode_set_state(g_ode, soa), "state upload");
        free(soa);
        g_ode_cells = n;
    }
    if (n != g_ode_cells) {
        fprintf(stderr, "monoalg3d_b200 shim: the number of cells changed\n");
        exit(1);
    }
    /* V (every neq-th value of sv) through a contiguous buffer; the strided
     * gather and scatter use the host's threads (the reference's own OpenMP
     * team size) */
    if (!g_vbuf) {
        g_vbuf = (double *)malloc((size_t)n * sizeof(double));
        if (!g_vbuf) {
            fprintf(stderr, "monoalg3d_b200 shim: out of host memory\n");
            exit(1);
        }
    }
    const real *sv = ode_solver->sv;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) g_vbuf[i] = sv[(size_t)i * neq];
    shim_check(mb_ode_set_v(g_ode, g_vbuf, 1), "V upload");
    shim_check(mb_solve_model_odes_gpu(g_ode, current_t, stim_currents), "solve_model_odes");
    shim_check(mb_ode_get_v(g_ode, g_vbuf, 1), "V download");
    real *svw = ode_solver->sv;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) svw[(size_t)i * neq] = g_vbuf[i];
}

/* ---- GPU build: the state lives on the device (ode_solver.h:37-47) -------- */

SET_ODE_INITIAL_CONDITIONS_GPU(set_model_initial_conditions_gpu) {
    (void)ode_extra_config;
    if (solver->adaptive || solver->cells_to_solve) {
        fprintf(stderr, "monoalg3d_b200 shim: adaptive meshes and the adaptive ODE step are not supported\n");
        exit(1);
    }
    const uint32_t n = solver->original_num_cells;
    free(g_celltype);
    g_celltype = torord_celltypes(solver, n);
    if (g_ode) mb_ode_destroy(g_ode);
    /* num_steps is set by the host after this call; the first solve updates it */
    shim_check(mb_ode_create(&g_ode, MB_SHIM_MODEL, MB_PREC_FP64, MB_RL_REFERENCE_CPU, n, solver->min_dt, 1),
               "mb_ode_create");
    size_t pitch = 0;
    shim_check(mb_set_model_initial_conditions_gpu(g_ode, NULL, g_celltype, &pitch), "initial conditions");
    double *sv = NULL;
    shim_check(mb_ode_device_state(g_ode, &sv, &pitch), "device state");
    solver->sv = (real *)sv;      /* freed by the host with cudaFree at exit (ode_solver.c:45-49) */
    g_ode_cells = n;
    return pitch;
}

SOLVE_MODEL_ODES(solve_model_odes_gpu) {
    (void)ode_extra_config;
    if (!g_ode || (uint32_t)ode_solver->num_cells_to_solve != g_ode_cells) {
        fprintf(stderr, "monoalg3d_b200 shim: solve_model_odes_gpu before set_model_initial_conditions_gpu, or the "
                        "number of cells changed\n");
        exit(1);
    }
    shim_check(mb_ode_set_steps(g_ode, ode_solver->min_dt, ode_solver->num_steps), "num_steps");
    shim_check(mb_solve_model_odes_gpu(g_ode, current_t, stim_currents), "solve_model_odes_gpu");
}

/* ---- linear system solver (linear_system_solver_config.h:12-21) ---------- */

static mb_csr *g_csr;
static uint32_t g_rows;
static double *g_b, *g_x;
static double g_tol = 1e-16;
static int g_max_its = 200;
static int g_precond = 0;

static const char *config_value(struct config *config, const char *key) {
    if (!config || !config->config_data) return NULL;
    for (ptrdiff_t i = 0; i < shlen(config->config_data); ++i)
        if (config->config_data[i].key && strcmp(config->config_data[i].key, key) == 0)
            return config->config_data[i].value;
    return NULL;
}

static int truthy(const char *v) {
    return v && (strcmp(v, "yes") == 0 || strcmp(v, "true") == 0 || strcmp(v, "1") == 0);
}

INIT_LINEAR_SYSTEM(init_conjugate_gradient) {
    (void)the_grid;
    if (is_purkinje) {
        fprintf(stderr, "monoalg3d_b200 shim: Purkinje systems are not supported\n");
        exit(1);
    }
    const char *v;
    if ((v = config_value(config, "tolerance"))) g_tol = strtod(v, NULL);
    if ((v = config_value(config, "max_iterations"))) g_max_its = atoi(v);
    g_precond = truthy(config_value(config, "use_preconditioner"));
}

static void upload_matrix(uint32_t n, struct cell_node **cells) {
    int32_t *row_ptr = (int32_t *)malloc(((size_t)n + 1) * sizeof(int32_t));
    size_t nnz = 0;
    for (uint32_t i = 0; i < n; ++i) nnz += (size_t)arrlen(cells[i]->elements);
    if (nnz > (size_t)INT32_MAX) {
        fprintf(stderr, "monoalg3d_b200 shim: more than 2^31 - 1 matrix entries\n");
        exit(1);
    }
    int32_t *col = (int32_t *)malloc((nnz ? nnz : 1) * sizeof(int32_t));
    double *val = (double *)malloc((nnz ? nnz : 1) * sizeof(double));
    g_b = (double *)malloc((size_t)n * sizeof(double));
    g_x = (double *)malloc((size_t)n * sizeof(double));
    if (!row_ptr || !col || !val || !g_b || !g_x) {
        fprintf(stderr, "monoalg3d_b200 shim: out of host memory\n");
        exit(1);
    }
    row_ptr[0] = 0;
    for (uint32_t i = 0; i < n; ++i) row_ptr[i + 1] = row_ptr[i] + (int32_t)arrlen(cells[i]->elements);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const struct element *el = cells[i]->elements;
        const int32_t k0 = row_ptr[i], m = row_ptr[i + 1] - k0;
        for (int32_t e = 0; e < m; ++e) {
            col[k0 + e] = (int32_t)el[e].column;
            val[k0 + e] = el[e].value;
        }
    }
    shim_check(mb_csr_create(&g_csr, (int32_t)n, row_ptr, col, val), "matrix upload");
    g_rows = n;
    free(row_ptr);
    free(col);
    free(val);
}

SOLVE_LINEAR_SYSTEM(conjugate_gradient) {
    (void)time_info;
    (void)config;
    (void)the_grid;
    if (!g_csr) upload_matrix(num_active_cells, active_cells);
    if (num_active_cells != g_rows) {
        fprintf(stderr, "monoalg3d_b200 shim: the matrix changed size (adaptivity is not supported)\n");
        exit(1);
    }
    /* b and the initial guess out of the host's cells, the solution back
     * into them, on the host's threads */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)num_active_cells; ++i) {
        g_b[i] = active_cells[i]->b;
        g_x[i] = active_cells[i]->v;
    }
    uint32_t its = 0;
    double err = 0.0;
    shim_check(mb_csr_solve(g_csr, g_b, g_x, g_tol, g_max_its, g_precond, &its, &err), "conjugate_gradient");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)num_active_cells; ++i) active_cells[i]->v = g_x[i];
    *number_of_iterations = its;
    *error = err;
}

END_LINEAR_SYSTEM(end_conjugate_gradient) {
    (void)config;
    mb_csr_destroy(g_csr);
    g_csr = NULL;
    free(g_b);
    free(g_x);
    g_b = g_x = NULL;
    g_rows = 0;
}

/* CPU restatement of MonoAlg3D's operator-split monodomain step, in plain C
 * and FP64 -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker for the CUDA path: the tests, the smoke check
 * and the CPU-baseline leg of bench.py call it; nothing in the product links
 * or loads it.  Each function names the reference file:line it restates
 * (paths relative to the MonoAlg3D_C source tree).  It is pinned against the
 * reference's own CPU build on the golden fixtures under tests/golden/.
 *
 * The tissue is described with the product's mb_monodomain_desc so a test can
 * hand the same description to both; only the FP64 fields are used
 * (precision is ignored: the oracle is always FP64).
 */
#ifndef MB_ORACLE_H
#define MB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "monoalg3d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- cell models (one cell, AoS state) ---------------------------------- */

#define ORC_TT_NEQ 19
#define ORC_TOR_NEQ 43

/* Default initial state of ten Tusscher 2006 (ten_tusscher_2006_RS_CPU.c:27-45). */
void orc_tt2006_initial_state(double *sv);
/* One Rush-Larsen sub-step of one cell (ten_tusscher_2006_RS_CPU.c:100-134 with
 * RHS_cpu :137-351); scale = 5 conductance multipliers (gNa, gKr, gKs, gCaL,
 * gK1) or NULL. */
void orc_tt2006_step(double *sv, double stim, double dt, const double *scale);

/* Steady-state initial state of ToRORd-fkatp for celltype 0 endo / 1 mid /
 * 2 epi (ToRORd_fkatp_mixed_endo_mid_epi.c:38-154). */
void orc_torord_initial_state(int celltype, double *sv);
/* One sub-step of one cell (ToRORd_fkatp_mixed_endo_mid_epi.c:252-310 with
 * RHS_RL_cpu :718-791 and _RL.common.c); rl_rule = enum mb_rl_rule. */
void orc_torord_step(double *sv, double stim, double dt, int celltype, int rl_rule, const double *scale);

/* ---- assembly, linear solver -------------------------------------------- */

/* CSR matrix of (alpha I + K) over the active cells in grid order. */
typedef struct orc_csr {
    int32_t n;           /* active cells                                     */
    int32_t *row_ptr;    /* n + 1                                            */
    int32_t *col;        /* nnz, diagonal first in each row                  */
    double *val;
} orc_csr;

/* Assembles the tissue's matrix: homogeneous_sigma_assembly_matrix
 * (matrix_assembly.c:334-387, assembly_common.c:4-78,911-1048) or
 * anisotropic_sigma_assembly_matrix (matrix_assembly.c:389-514,
 * assembly_common.c:115-412,437-908,1102-1139).  cells[] receives the grid
 * index of every row.  Returns 0 or an MB_ERR_* code. */
int orc_assemble(const mb_monodomain_desc *d, orc_csr *A, int32_t *cells);
void orc_csr_free(orc_csr *A);

/* cpu_conjugate_gradient (linear_system_solver.c:47-183) on a CSR matrix
 * whose first entry in each row is the diagonal. */
void orc_pcg(const orc_csr *A, const double *b, double *x, double tol, int max_its, int use_preconditioner,
             uint32_t *its, double *error);

/* ---- the time loop ------------------------------------------------------ */

typedef struct orc_sim orc_sim;

int orc_create(orc_sim **out, const mb_monodomain_desc *d);
/* Runs nsteps iterations of solve_monodomain's loop body
 * (monodomain_solver.c:616-925 without output and ECG). */
int orc_step(orc_sim *s, int nsteps);
/* V over the grid (removed cells NaN). */
void orc_get_v(const orc_sim *s, double *v_grid);
/* State variable `var` of every active cell, in grid order. */
void orc_get_state(const orc_sim *s, int var, double *out);
/* CG iterations / error of the last step; total steps taken; current time. */
void orc_last_cg(const orc_sim *s, uint32_t *its, double *error);
double orc_time(const orc_sim *s);
int32_t orc_active_cells(const orc_sim *s);
void orc_destroy(orc_sim *s);
/* Loop steps the reference takes for final time T (cur_time - T <= dt). */
int orc_loop_steps(double final_time, double dt);
/* Per-row stimulus values of every stimulus (num_stims x n), for the rows
 * whose grid indices are cells[] (stimuli.c:56-91,426-520). */
void orc_stim_values(const mb_monodomain_desc *d, const int32_t *cells, int32_t n, double *out);

/* ---- tangent-linear loop (tangent.cc) ----------------------------------- */

/* Runs nsteps loop steps of a TT2006 tissue with per-cell conductivity
 * (MB_ASSEMBLY_PER_CELL_SIGMA) and samples V at the sensor cells (grid
 * indices) after every sample_every steps.  Returns the L2 misfit
 * loss = 1/2 sum (sample - target)^2 (target: nsteps / sample_every rows of
 * n_sensors) and its derivative dloss along the direction (dsigma, dgkr):
 * per grid cell, a change of the conductivity and of the gKr scaling (either
 * may be NULL).  Forward mode: the cell model runs orc_tt2006_step's
 * statements on dual numbers, and every implicit solve A v = b is followed by
 * the tangent solve A dv = alpha dV* - dA v, dA from the derivative of the
 * harmonic-mean face conductivities.  Returns 0 or an MB_ERR_* code. */
int orc_tangent_misfit(const mb_monodomain_desc *d, int nsteps, int sample_every, int n_sensors,
                       const int64_t *sensors, const double *target, const double *dsigma, const double *dgkr,
                       double *loss, double *dloss);

#ifdef __cplusplus
}
#endif
#endif

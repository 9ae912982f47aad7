/*
 * monoalg3d_b200.h -- C ABI of the B200-native monodomain step.
 *
 * One operator-split monodomain time step of MonoAlg3D on a fixed structured
 * mesh, run entirely on one GPU:
 *
 *   1. Rush-Larsen ionic ODEs (ten Tusscher 2006, ToRORd-fkatp endo/mid/epi),
 *   2. the update_monodomain right-hand side b = alpha * V*,
 *   3. a Jacobi-preconditioned CG solve of (alpha I + K) V = b,
 *
 * exactly in the order of the reference time loop
 * (src/monodomain/monodomain_solver.c:616-925).  Every entry point takes plain
 * pointers and sizes; host buffers are ordinary C arrays.  All functions return
 * an int status: MB_OK (0) or one of the MB_ERR_* codes; mb_last_error()
 * returns a readable message for the calling thread's last failure.
 *
 * Entry points and the reference plugin functions they replace:
 *
 *   mb_init_cell_model_data            init_cell_model_data
 *                                      (src/ode_solver/ode_solver.h:33,
 *                                       ten_tusscher_2006_RS_CPU.c:5-14,
 *                                       ToRORd_fkatp_mixed_endo_mid_epi.c:4-10)
 *   mb_ode_create +
 *   mb_set_model_initial_conditions_gpu set_model_initial_conditions_gpu
 *                                      (ode_solver.h:46; returns the pitch)
 *   mb_solve_model_odes_gpu            solve_model_odes_gpu (ode_solver.h:37;
 *                                      stim_currents is a host array as in
 *                                      ode_solver.c:183-248)
 *   mb_monodomain_create               set_initial_conditions_fvm +
 *                                      homogeneous_sigma_assembly_matrix /
 *                                      anisotropic_sigma_assembly_matrix
 *                                      (matrix_assembly.c:27-45,334-514) and
 *                                      init_conjugate_gradient
 *                                      (linear_system_solver.c:202-216)
 *   mb_update_monodomain_default       update_monodomain_default
 *                                      (update_monodomain.c:19-56)
 *   mb_conjugate_gradient              conjugate_gradient
 *                                      (linear_system_solver.c:185-200)
 *   mb_monodomain_step                 one pass of the solve_monodomain loop
 *                                      body (monodomain_solver.c:616-925)
 *   mb_csr_conjugate_gradient          cpu_conjugate_gradient /
 *                                      gpu_conjugate_gradient on a matrix read
 *                                      from file (test_solvers.c:28-111)
 *   mb_monodomain_destroy              end_conjugate_gradient + free of sv
 *
 * Threading: every object is used from one host thread at a time, as the
 * reference plugins are (one solver configuration per process there; one per
 * object here).
 */
#ifndef MONOALG3D_B200_H
#define MONOALG3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MB_OK               0
#define MB_ERR_ARG          1   /* invalid argument                         */
#define MB_ERR_CUDA         2   /* a CUDA runtime call failed               */
#define MB_ERR_NAN          3   /* NaN in the CG error (monodomain_solver.c:746) */
#define MB_ERR_NOMEM        4   /* host or device allocation failed         */
#define MB_ERR_UNSUPPORTED  5   /* combination not implemented              */
#define MB_ERR_STATE        6   /* object used in the wrong order           */

/* ---- enumerations ------------------------------------------------------ */
enum mb_model {
    MB_MODEL_TT2006 = 0,               /* libten_tusscher_2006, 19 states    */
    MB_MODEL_TORORD_FKATP_MIXED = 1,   /* libToRORd_fkatp_mixed_endo_mid_epi, 43 states */
    MB_MODEL_TORORD_FKATP_ENDO = 2     /* libToRORd_fkatp_endo, 43 states, forward Euler
                                          (fixed or adaptive step, see ode_adaptive) */
};

enum mb_precision {
    MB_PREC_FP64 = 0,   /* FP64 everywhere (the plain method)                  */
    MB_PREC_MIXED = 1   /* FP32 ODE with FP64 ion concentrations; FP32 CG with
                           FP64 solution, FP64 dot accumulation and FP64
                           true-residual refinement                              */
};

/* How a Rush-Larsen gate of the ToRORd model picks its branch
 * (ToRORd_fkatp_mixed_endo_mid_epi.h:20).  The reference CPU build applies C
 * abs() to a double, which truncates to int: every gate with |a| < 1 takes the
 * explicit Euler branch.  MB_RL_TRUE uses |a| < 1e-8 as written.            */
enum mb_rl_rule {
    MB_RL_REFERENCE_CPU = 0,
    MB_RL_TRUE = 1
};

enum mb_stim_kind {
    MB_STIM_X_LESS_THAN = 0,   /* stim_if_x_less_than  (stimuli.c:56-91)    */
    MB_STIM_X_Y_LIMITS = 1,    /* stim_x_y_limits      (stimuli.c:426-467)  */
    MB_STIM_X_Y_Z_LIMITS = 2,  /* stim_x_y_z_limits    (stimuli.c:469-520)  */
    MB_STIM_CELL_MASK = 3      /* explicit per-cell mask given by the caller */
};

enum mb_assembly {
    /* homogeneous_sigma_assembly_matrix (matrix_assembly.c:334-387): 7-point,
       harmonic-mean face conductivities                                     */
    MB_ASSEMBLY_HOMOGENEOUS = 0,
    /* anisotropic_sigma_assembly_matrix (matrix_assembly.c:389-514) with a
       per-z-plane fibre direction in the xy plane: 19-point stencil         */
    MB_ASSEMBLY_ANISOTROPIC = 1,
    /* per-cell isotropic sigma, harmonic mean per face (7-point)            */
    MB_ASSEMBLY_PER_CELL_SIGMA = 2
};

#define MB_MAX_STIMS 8

typedef struct mb_stim {
    int    kind;        /* enum mb_stim_kind                                 */
    double start;       /* ms                                                */
    double duration;    /* ms; active for start <= t <= start + duration     */
    double period;      /* ms; 0 = not periodic (ode_solver.c:225-233)       */
    double current;     /* uA/uF, added to dV/dt with a minus sign           */
    double x_limit;     /* MB_STIM_X_LESS_THAN: center.x < x_limit (um)      */
    double min[3];      /* MB_STIM_X_Y(_Z)_LIMITS: inclusive box on centers  */
    double max[3];
    const uint8_t *cell_mask; /* MB_STIM_CELL_MASK: nx*ny*nz bytes, 1 = stim */
} mb_stim;

/* Description of one tissue on a structured cuboid grid.  Cell (i,j,k) has
 * centre ((i+1/2)dx, (j+1/2)dy, (k+1/2)dz) um, as set_cuboid_domain_mesh
 * builds it (domain_helpers.c:19-73); grid index is i + nx*(j + ny*k).      */
typedef struct mb_monodomain_desc {
    int    nx, ny, nz;
    double dx, dy, dz;                 /* um                                  */
    const uint8_t *active;             /* nx*ny*nz bytes, 0 = removed cell;
                                          NULL = every cell active            */
    /* [main] */
    double dt_pde;                     /* ms                                  */
    double beta;                       /* 1/um   (default 0.14)               */
    double cm;                         /* uF/cm^2 (default 1.0)               */
    /* [ode_solver] */
    int    model;                      /* enum mb_model                       */
    int    precision;                  /* enum mb_precision                   */
    int    rl_rule;                    /* enum mb_rl_rule (ToRORd only)       */
    double dt_ode;                     /* ms; num_steps = (int)(dt_pde/dt_ode) */
    const double *initial_state;       /* NEQ values for every cell, or NULL
                                          for the model defaults              */
    const uint8_t *celltype;           /* ToRORd: nx*ny*nz bytes, 0 endo,
                                          1 mid, 2 epi; NULL = all endo       */
    const double *current_scale;       /* per-cell conductance scalings,
                                          MB_NUM_SCALES x (nx*ny*nz), row
                                          major by scale; NULL = all 1; kept
                                          and applied as float values         */
    /* [assembly_matrix] */
    int    assembly;                   /* enum mb_assembly                    */
    double sigma[3];                   /* homogeneous: sigma_x, sigma_y, sigma_z (mS/um) */
    double sigma_l, sigma_t, sigma_n;  /* anisotropic: along / across fibres  */
    const double *fibre_angle_z;       /* anisotropic: nz angles (rad) of the
                                          fibre in the xy plane, NULL = 0     */
    const double *sigma_cell;          /* per-cell sigma (nx*ny*nz), PER_CELL */
    /* [linear_system_solver] */
    double cg_tolerance;               /* stop when r.r <= tolerance          */
    int    cg_max_iterations;          /* default 200                         */
    int    use_preconditioner;         /* Jacobi                              */
    /* [stim_*] */
    int    num_stims;
    mb_stim stims[MB_MAX_STIMS];
    /* initial transmembrane potential for the CG initial guess
       (set_initial_conditions_fvm, matrix_assembly.c:27-45);
       NaN = the model's INITIAL_V                                          */
    double initial_v;
    /* activation time / APD90 per active cell, tracked on the device (see
       mb_monodomain_get_activation); 0 = off                               */
    int    track_activation;
    double activation_threshold;       /* mV, default -30                     */
    double activation_min_interval;    /* ms, default 10                      */
    /* [calc_ecg] pseudo_bidomain (ecg_library/ecg.c:204-307): at the start
       of every step whose count is a multiple of ecg_rate, from the V of
       that moment; 0 = off.  Electrodes at ecg_leads (3 per lead, um, in
       the grid's frame: cell (i,j,k) is centred at ((i+1/2)dx, ...)), at
       most MB_ECG_MAX_LEADS; records kept on the device, at most
       ecg_capacity (read with mb_monodomain_get_ecg).                      */
    int    ecg_rate;
    int    ecg_n_leads;
    const double *ecg_leads;
    double ecg_sigma_b;                /* bath conductivity, sigma_b of the reference */
    int64_t ecg_capacity;
    /* [ode_solver] adaptive = true, for the forward-Euler library
       (MB_MODEL_TORORD_FKATP_ENDO; default_solvers.c:55-175): each cell
       steps with its own error-controlled dt in [min_dt, max_dt], min_dt =
       dt_ode (the reference takes 1e-10 when no dt is given,
       ode_solver.c:311-328), max_dt = dt_pde, tolerances ode_abs_tol /
       ode_rel_tol (default 1e-5).  Each
       loop step integrates every cell up to cur_time + min_dt
       (MB_ODE_ADAPTIVE_CPU, the CPU build's solve_model_odes_cpu) or up to
       cur_time + max_dt (MB_ODE_ADAPTIVE_GPU, the GPU build's solve_gpu).   */
    int    ode_adaptive;               /* enum mb_ode_adaptive                */
    double ode_abs_tol, ode_rel_tol;
} mb_monodomain_desc;

enum mb_ode_adaptive {
    MB_ODE_FIXED = 0,
    MB_ODE_ADAPTIVE_CPU = 1,
    MB_ODE_ADAPTIVE_GPU = 2
};

#define MB_ECG_MAX_LEADS 16

/* Scalings of the ionic conductances, in this order (TT2006: gNa, gKr, gKs,
 * gCaL, gK1; ToRORd: the same currents).                                    */
#define MB_NUM_SCALES 5

typedef struct mb_monodomain mb_monodomain;
typedef struct mb_ode mb_ode;

/* Per-step record kept on the device: CG iterations and final r.r. */
typedef struct mb_step_stats {
    int32_t cg_iterations;
    int32_t refinements;     /* FP64 true-residual evaluations (mixed)      */
    double  cg_error;
} mb_step_stats;

/* ---- errors / device --------------------------------------------------- */
const char *mb_last_error(void);
int mb_version(void);
int mb_device_count(int *count);

/* ---- cell model library (ode_solver.h:33-47) --------------------------- */
int mb_init_cell_model_data(int model, int *number_of_ode_equations, double *initial_v);
/* Initial state of the ToRORd_fkatp_endo library (43 values): its CPU
 * build's (ToRORd_fkatp_endo.c:30-76, the default of a tissue) or, with
 * gpu_build, its GPU build's, a different steady state
 * (ToRORd_fkatp_endo.cu:8-50); pass the latter as initial_state to follow
 * the GPU build.                                                            */
int mb_torord_endo_initial_state(int gpu_build, double *state);
/* Default initial state of the ToRORd_fkatp_mixed_endo_mid_epi library for
 * a cell type (0 endo, 1 mid, 2 epi; 43 values): the steady states it and
 * the ToRORd extra data tabulate (ToRORd_fkatp_mixed_endo_mid_epi.c:110-154,
 * helper_functions.c:166-300).                                              */
int mb_torord_initial_state(int celltype, double *state);

/* Stand-alone ODE object: num_cells independent cells, state in SoA rows. */
int mb_ode_create(mb_ode **out, int model, int precision, int rl_rule,
                  uint32_t num_cells, double dt, uint32_t num_steps);
/* Writes the initial state; initial_state = NULL uses the model defaults,
 * celltype = NULL makes every cell ENDO.  *pitch_out = bytes between state
 * rows, as the reference returns from set_model_initial_conditions_gpu.    */
int mb_set_model_initial_conditions_gpu(mb_ode *ode, const double *initial_state,
                                        const uint8_t *celltype, size_t *pitch_out);
/* num_steps sub-steps of size dt for every cell; stim_currents[num_cells]
 * is read from host memory (NULL = no stimulus).                          */
int mb_solve_model_odes_gpu(mb_ode *ode, double current_t, const double *stim_currents);
/* Copies the state, neq rows of num_cells doubles, to host memory. */
int mb_ode_get_state(mb_ode *ode, double *host_state);
int mb_ode_set_state(mb_ode *ode, const double *host_state);
/* V alone (state 0 of every cell) from / to host memory with an element
 * stride; stride = number_of_ode_equations reads and writes the reference's
 * CPU state vector sv[i * neq] in place (what the orchestrator writes before
 * solve_model_odes_cpu and update_monodomain_default reads after it,
 * monodomain_solver.c:1051, update_monodomain.c:50).                       */
int mb_ode_set_v(mb_ode *ode, const double *v, size_t stride);
int mb_ode_get_v(mb_ode *ode, double *v, size_t stride);
/* The device state itself: *sv = row 0 of the FP64 state rows (V, then the
 * other states, one row of num_cells values every *pitch bytes), the pitched
 * array the reference's GPU build keeps in ode_solver->sv and reads and
 * writes row 0 of (update_ode_state_vector, monodomain_solver.c:1026-1045;
 * update_monodomain.c:31-52).  FP64 objects only.                          */
int mb_ode_device_state(mb_ode *ode, double **sv, size_t *pitch);
/* Changes the sub-step size and count of later solves (the reference sets
 * num_steps after the initial conditions, monodomain_solver.c:512-520).    */
int mb_ode_set_steps(mb_ode *ode, double dt, uint32_t num_steps);
void mb_ode_destroy(mb_ode *ode);

/* ---- monodomain tissue ------------------------------------------------- */
void mb_monodomain_desc_defaults(mb_monodomain_desc *d);
int  mb_monodomain_create(mb_monodomain **out, const mb_monodomain_desc *desc);
void mb_monodomain_destroy(mb_monodomain *m);

/* Runs n loop iterations of solve_monodomain (ODE, RHS, CG, clock) on the
 * device; asynchronous with respect to the host.                          */
int mb_monodomain_step(mb_monodomain *m, int n);
/* Waits for the device, then checks the NaN flag. */
int mb_monodomain_sync(mb_monodomain *m);

/* The three phases one at a time, for callers that drive the loop
 * themselves the way monodomain_solver.c does.                            */
int mb_solve_all_volumes_odes(mb_monodomain *m);
int mb_update_monodomain_default(mb_monodomain *m);
int mb_conjugate_gradient(mb_monodomain *m, uint32_t *number_of_iterations, double *error);
int mb_advance_time(mb_monodomain *m);

/* Reference-host mode: per step, take the stimulus from a host array, run
 * ODE + RHS + CG and return V to host memory -- the copies the reference GPU
 * plugins make every step (monodomain_solver.c:1012-1105,
 * update_monodomain.c:35-38).  stim_host may be NULL.                     */
int mb_monodomain_step_host(mb_monodomain *m, const double *stim_host, double *v_host);

/* State access (host buffers, grid order nx*ny*nz; removed cells get NaN). */
int mb_monodomain_get_v(mb_monodomain *m, double *v_host);
int mb_monodomain_set_v(mb_monodomain *m, const double *v_host);
int mb_monodomain_get_state(mb_monodomain *m, double *state_host);  /* NEQ x n_active */
int mb_monodomain_info(mb_monodomain *m, int64_t *count, double *cur_time,
                       uint32_t *n_active, int *neq);
int mb_monodomain_step_stats(mb_monodomain *m, int64_t first, int64_t n, mb_step_stats *out);
/* Activation times per grid cell, tracked on the device at every loop step
 * (needs track_activation): an activation is an upward crossing of
 * activation_threshold at least activation_min_interval after the previous
 * one (the rules of save_with_activation_times, save_mesh.c:754-913), its
 * time linearly interpolated between the two loop steps; APD90 runs from it
 * to the downward crossing of V_peak - 0.9 (V_peak - V_rest), also
 * interpolated.  first / last: first and latest activation time (ms),
 * apd90: APD90 of the latest beat (ms), count: activations.  Cells never
 * activated, beats not yet repolarised and removed cells read -1 (count 0).
 * Any pointer may be NULL.                                                  */
int mb_monodomain_get_activation(mb_monodomain *m, float *first, float *last, float *apd90, int32_t *count);

/* ECG records taken so far (*records), and records first .. first+n-1 of
 * them: times[n] (ms, the loop clock of the step) and values[n x n_leads]
 * (lead after lead, the reference's ecg.txt columns: -1/(4 pi sigma_b)
 * sum over active cells of beta_im vol / |x - lead|, ecg.c:264-307).
 * Either array may be NULL.                                                */
int mb_monodomain_get_ecg(mb_monodomain *m, int64_t first, int64_t n, double *times, double *values,
                          int64_t *records);

/* ---- batches of independent tissues ------------------------------------
 * No counterpart in the reference (which runs one tissue per process).  The
 * n tissues, tissue i a 2-D sheet nx[i] x ny[i] (ny[i] = 1: a cable), are
 * placed side by side in one 2-D atlas grid with removed cells between them,
 * so that no face couples two tissues; the atlas is then solved as one
 * tissue (one ODE launch, one persistent CG launch and one graph replay per
 * step for the whole batch), with per-tissue parameters given as per-cell
 * arrays.  Tissue i occupies atlas cells (x0[i] + i', y0[i] + j') for
 * 0 <= i' < nx[i], 0 <= j' < ny[i].  Shelf packing, tallest first.          */
int mb_batch_pack(int n, const int *nx, const int *ny, int *atlas_nx, int *atlas_ny, int *x0, int *y0);

/* ---- discrete adjoint ----------------------------------------------------
 * No counterpart in the reference.  Gradient of a scalar function of the V
 * traces at sensor cells with respect to the per-cell conductivity and the
 * per-cell gKr scaling, by the discrete adjoint of the loop: the transposed
 * Jacobian of each Rush-Larsen step and a transposed (here: the same,
 * symmetric) PCG solve per step, run backwards over checkpoints of the loop
 * state taken every checkpoint_every steps, the states in between recomputed.
 * The tissue (d) must be ten Tusscher 2006, FP64, per-cell conductivity
 * (MB_ASSEMBLY_PER_CELL_SIGMA), with conductance scalings and dt_ode = dt_pde.
 * Samples: V at the sensors after every sample_every steps
 * (nsteps / sample_every samples).                                          */
typedef struct mb_adjoint mb_adjoint;
int mb_adjoint_create(mb_adjoint **out, const mb_monodomain_desc *d, int nsteps, int checkpoint_every,
                      int n_sensors, const int64_t *sensor_cells, int sample_every);
/* Runs the loop from the initial state with new conductivities and scalings
 * (grid order; NULL keeps the current ones); traces: samples x sensors.      */
int mb_adjoint_forward(mb_adjoint *a, const double *sigma_cell, const double *scale, double *traces);
/* Given dL/dtraces (samples x sensors), the gradients with respect to
 * sigma_cell and to the gKr scaling (row 1 of the scalings), grid order.     */
int mb_adjoint_backward(mb_adjoint *a, const double *dtraces, double *grad_sigma, double *grad_scale_gkr);
void mb_adjoint_destroy(mb_adjoint *a);

/* Checkpoint / restore of the whole loop state (V, V*, the ODE state rows,
 * the clock and stimulus table, activation tracking) to host memory in this
 * library's own layout, for a tissue of the same shape, model and precision
 * (the reference's layout: mb_monodomain_save_state below).                 */
int mb_monodomain_checkpoint_bytes(mb_monodomain *m, size_t *bytes);
int mb_monodomain_checkpoint(mb_monodomain *m, void *host, size_t bytes);
int mb_monodomain_restore(mb_monodomain *m, const void *host, size_t bytes);
/* Checkpoints in the reference's own layout: the three files of
 * save_simulation_state (src/save_state_library/save_state.c:16-150) --
 * grid_checkpoint.dat, monodomain_solver_checkpoint.dat and
 * ode_solver_checkpoint.dat -- in the directory dir, which
 * restore_simulation_state (restore_state.c:38-230) reads back into the
 * reference's own loop, and which mb_monodomain_restore_state reads from the
 * reference's.  The state vector is written in the reference's numbering of
 * the active cells (the Hilbert order of its octree) and, with gpu_layout,
 * state row after state row as its GPU build writes it (with the row pitch
 * cudaMallocPitch gives on this device), else cell after cell as its CPU
 * build does.  Restore checks the mesh, active cell count, dt, beta and cm
 * against the tissue's and sets V, the ODE state and the loop clock (step
 * count, time); activation tracking and the ECG records are not part of the
 * layout.  Cell centres are matched exactly, as the reference matches them:
 * spacings whose half-integer multiples are exact in double (100 um) are
 * supported.                                                                 */
int mb_monodomain_save_state(mb_monodomain *m, const char *dir, int gpu_layout);
int mb_monodomain_restore_state(mb_monodomain *m, const char *dir);
/* The reference's numbering of the active cells of an nx x ny x nz cuboid
 * with an optional removed-cell mask (grid order, 0 = removed): order[r] =
 * grid index of active cell r (order_grid_cells, grid.c:245-263, over the
 * octree of set_cuboid_domain_mesh, domain_helpers.c:19-73); also the number
 * of active cells and of all the octree's leaves.  Host only.  Any output
 * may be NULL.                                                              */
int mb_reference_cell_order(int nx, int ny, int nz, const uint8_t *active, int64_t *order, int64_t *n_active,
                            int64_t *number_of_cells);
/* V of the active cells in the format of save_as_text_or_binary
 * (save_mesh.c:248-420): "x,y,z,hx,hy,hz,V" per line, or 7 doubles per cell
 * when binary; cells in grid order.                                          */
int mb_monodomain_save_v(mb_monodomain *m, const char *path, int binary);

/* Device pointers to V (double, grid order) and to the CUDA stream used.
 * V may be written through the pointer between steps (stream-ordered); the
 * next mixed z-march solve, which otherwise starts from the product A x its
 * previous solve stored, then takes more iterations to reach the same
 * tolerance (mb_monodomain_set_v tells the tissue instead).               */
int mb_monodomain_device_v(mb_monodomain *m, double **v_dev, void **stream);
/* Average duration of the last kernel launches per kind, from CUDA events
 * recorded by mb_monodomain_profile_steps: ode, cg (whole solve). */
int mb_monodomain_profile_steps(mb_monodomain *m, int n, double *ode_ms, double *cg_ms,
                                double *step_ms, int *cg_iterations);

/* Device time (CUDA events on the tissue's stream) of n whole steps, and of n
 * reference-host steps (mb_monodomain_step_host with the given buffers).    */
int mb_monodomain_time_steps(mb_monodomain *m, int n, double *ms);
int mb_monodomain_time_steps_host(mb_monodomain *m, int n, const double *stim_host, double *v_host,
                                  double *ms);

/* Pipelined reference-host steps (no reference counterpart; the same work
 * and copies as mb_monodomain_step_host): call k copies its stimulus in and
 * its V out on a copy stream that runs under the compute of the neighbouring
 * steps, and returns once the copies of call k - 1 are done (its V is in its
 * host buffer, its buffers may be refilled), so the caller alternates two
 * pairs of host buffers (pinned, for the copies to overlap).
 * mb_monodomain_host_wait completes the last call's copies.  The timed form
 * runs n steps with buffer pairs (stim0, v0) and (stim1, v1) and reports the
 * device time from the first copy to the last.                             */
int mb_monodomain_step_host_async(mb_monodomain *m, const double *stim_host, double *v_host);
int mb_monodomain_host_wait(mb_monodomain *m);
int mb_monodomain_time_steps_host_async(mb_monodomain *m, int n, const double *stim0, const double *stim1,
                                        double *v0, double *v1, double *ms);

/* Launch choices made at creation by timing: the ODE kernel's variant
 * (0..5 = one-cell-per-thread launches with at least 1..6 resident 128-thread
 * blocks per SM, 6..9 = staged persistent launches with at least 1..4), the
 * CG grid size and the CG kernel (-1 = graph of separate kernels, 0..n-1 =
 * launch shape of the flat persistent kernel, n = mb_cg_launch_shapes --
 * the first half with a contiguous range of cells per block, the second the
 * same shapes sweeping the grid interleaved --, 100 = the 2.5D tiled
 * persistent kernel, 200 = the resident tile-column kernel).  The
 * environment variable MB_CG_VARIANT, read at creation, forces a choice:
 * 0..n-1 a flat shape, n the tiled kernel, n + 1 the resident kernel. */
int mb_monodomain_tuning(mb_monodomain *m, int *ode_variant, int *cg_blocks, int *cg_kernel);
int mb_cg_launch_shapes(int *flat_shapes);

/* ---- general sparse CG (test_solvers.c fixtures) ---------------------- */
/* Solves A x = b for a CSR matrix on the device; x holds the initial guess
 * on entry.  Same iteration and stopping rule as cpu_conjugate_gradient
 * (linear_system_solver.c:47-183).                                         */
int mb_csr_conjugate_gradient(int32_t n, const int32_t *row_ptr, const int32_t *col,
                              const double *val, const double *b, double *x,
                              double tolerance, int max_iterations, int use_preconditioner,
                              uint32_t *number_of_iterations, double *error);

/* The same solver with the matrix kept on the device between solves: create
 * uploads it once, each solve copies b and x in and x out (the reference's
 * conjugate_gradient plugin call, linear_system_solver_config.h:12-16, on a
 * matrix assembled once).                                                  */
typedef struct mb_csr mb_csr;
int mb_csr_create(mb_csr **out, int32_t n, const int32_t *row_ptr, const int32_t *col, const double *val);
int mb_csr_solve(mb_csr *a, const double *b, double *x, double tolerance, int max_iterations,
                 int use_preconditioner, uint32_t *number_of_iterations, double *error);
void mb_csr_destroy(mb_csr *a);

/* ---- allocation-free CSR CG -------------------------------------------- */
/* No counterpart in the reference.  The same solve as
 * mb_csr_conjugate_gradient for callers that cannot allocate device memory
 * while they run (a host framework that owns all device memory through its
 * own pool, a real-time loop that cannot afford cudaMalloc's synchronisation,
 * a plugin handed device buffers by its host): row_ptr, col, val, b and x are
 * DEVICE pointers supplied by the caller, x holds the initial guess and
 * receives the solution, and the work vectors live in a fixed 16 MiB + 64 KiB
 * device array inside this library (held on every GPU that loads it until
 * exit; it is placed on a device, with the library's module, at the first call
 * made there, which may synchronise the device: make one warm-up call at
 * initialisation).  Nothing is allocated or freed.  n is limited to 524288
 * rows; larger systems are rejected with MB_ERR_ARG.  The array's device
 * address is looked up on that first call: make it before any stream capture
 * on the device.  Each call waits on its stream (it reads the convergence
 * flag back), which must belong to the current device.  All calls share the
 * array, so calls whose work overlaps on the GPU race and must be serialised
 * by the caller.  stream may be NULL (legacy default stream).  Returns the
 * iteration count and the final r.r in host memory.                          */
int mb_csr_conjugate_gradient_noalloc(int32_t n, const int32_t *row_ptr, const int32_t *col,
                                      const double *val, const double *b, double *x,
                                      double tolerance, int max_iterations, int use_preconditioner,
                                      uint32_t *number_of_iterations, double *error, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MONOALG3D_B200_H */

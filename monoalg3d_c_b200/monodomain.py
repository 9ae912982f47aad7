"""Host-side mirror of MonoAlg3D's monodomain plugin interface over the C ABI.

The names follow the reference plugins so that a driver script reads like
``solve_monodomain`` (src/monodomain/monodomain_solver.c:616-925):

    tissue.solve_all_volumes_odes()        # ode_solver.c:183-248
    tissue.update_monodomain_default()     # update_monodomain.c:19-56
    its, err = tissue.conjugate_gradient() # linear_system_solver.c:185-200
    tissue.advance_time()                  # monodomain_solver.c:907-908

``Tissue.step(n)`` runs n whole loop iterations as captured CUDA graphs.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import MbDesc, MbStepStats, MbStim, check, lib

MODELS = {"tt2006": _lib.MB_MODEL_TT2006, "ten_tusscher_2006": _lib.MB_MODEL_TT2006,
          "torord": _lib.MB_MODEL_TORORD_FKATP_MIXED,
          "ToRORd_fkatp_mixed_endo_mid_epi": _lib.MB_MODEL_TORORD_FKATP_MIXED,
          "torord_endo": _lib.MB_MODEL_TORORD_FKATP_ENDO, "ToRORd_fkatp_endo": _lib.MB_MODEL_TORORD_FKATP_ENDO}
ODE_ADAPTIVE = {None: _lib.MB_ODE_FIXED, "cpu": _lib.MB_ODE_ADAPTIVE_CPU, "gpu": _lib.MB_ODE_ADAPTIVE_GPU}
PRECISIONS = {"fp64": _lib.MB_PREC_FP64, "mixed": _lib.MB_PREC_MIXED}
RL_RULES = {"reference_cpu": _lib.MB_RL_REFERENCE_CPU, "true": _lib.MB_RL_TRUE}
ASSEMBLIES = {"homogeneous": _lib.MB_ASSEMBLY_HOMOGENEOUS, "anisotropic": _lib.MB_ASSEMBLY_ANISOTROPIC,
              "per_cell": _lib.MB_ASSEMBLY_PER_CELL_SIGMA}
STIM_KINDS = {"x_less_than": _lib.MB_STIM_X_LESS_THAN, "x_y_limits": _lib.MB_STIM_X_Y_LIMITS,
              "x_y_z_limits": _lib.MB_STIM_X_Y_Z_LIMITS, "cell_mask": _lib.MB_STIM_CELL_MASK}


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def init_cell_model_data(model: str):
    """(number_of_ode_equations, initial_v) of a cell model (init_cell_model_data)."""
    neq, v0 = C.c_int(), C.c_double()
    check(lib.mb_init_cell_model_data(MODELS[model], C.byref(neq), C.byref(v0)))
    return neq.value, v0.value


def torord_endo_initial_state(gpu_build: bool = False) -> np.ndarray:
    """The ToRORd_fkatp_endo library's initial state: its CPU build's (the
    tissue default) or its GPU build's (pass as initial_state to follow it)."""
    out = np.empty(43, dtype=np.float64)
    check(lib.mb_torord_endo_initial_state(1 if gpu_build else 0, out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def loop_steps(final_time: float, dt: float) -> int:
    """Iterations of ``while(cur_time - finalT <= dt_pde)`` with ``cur_time += dt_pde``
    accumulated in double, as the reference loop runs (monodomain_solver.c:616,908)."""
    cur, n = 0.0, 0
    while cur - final_time <= dt:
        n += 1
        cur += dt
    return n


@dataclass
class Stim:
    """One [stim_*] section: stim_if_x_less_than, stim_x_y_limits, stim_x_y_z_limits
    (stimuli.c:56-91,426-520) or an explicit per-cell mask."""
    kind: str = "x_less_than"
    start: float = 0.0
    duration: float = 2.0
    current: float = -53.0
    period: float = 0.0
    x_limit: float = 500.0
    min: Sequence[float] = (0.0, 0.0, 0.0)
    max: Sequence[float] = (0.0, 0.0, 0.0)
    cell_mask: Optional[np.ndarray] = None


def build_desc(nx: int, ny: int, nz: int, dx: float = 100.0, dy: float = 100.0, dz: float = 100.0, *,
               active: Optional[np.ndarray] = None, dt_pde: float = 0.02, dt_ode: Optional[float] = None,
               beta: float = 0.14, cm: float = 1.0, model: str = "tt2006", precision: str = "fp64",
               rl_rule: str = "reference_cpu", assembly: str = "homogeneous",
               sigma: Sequence[float] = (0.00013, 0.00013, 0.00013), sigma_l: float = 0.0,
               sigma_t: float = 0.0, sigma_n: Optional[float] = None,
               fibre_angle_z: Optional[np.ndarray] = None, sigma_cell: Optional[np.ndarray] = None,
               celltype: Optional[np.ndarray] = None, current_scale: Optional[np.ndarray] = None,
               initial_state: Optional[np.ndarray] = None, cg_tolerance: float = 1e-16,
               cg_max_iterations: int = 200, use_preconditioner: bool = True,
               stims: Sequence[Stim] = (), initial_v: float = float("nan"), track_activation: bool = False,
               activation_threshold: float = -30.0, activation_min_interval: float = 10.0,
               ecg_leads: Optional[Sequence[Sequence[float]]] = None, ecg_rate: int = 1, ecg_sigma_b: float = 1.0,
               ecg_capacity: int = 100000, ode_adaptive: Optional[str] = None, ode_abs_tol: float = 1e-5,
               ode_rel_tol: float = 1e-5) -> Tuple[MbDesc, list]:
    """The C-ABI tissue description (mb_monodomain_desc) for these arguments,
    with the arrays it points to (keep them alive while the description is
    in use).  Arrays given per cell are in grid order.  ode_adaptive ("cpu"
    or "gpu", forward-Euler model only) selects the adaptive ODE step with
    the reference CPU or GPU build's step end; its min_dt is dt_ode (1e-10
    when dt_ode is None, as the reference with no dt), max_dt is dt_pde."""
    n = nx * ny * nz
    d = MbDesc()
    lib.mb_monodomain_desc_defaults(C.byref(d))
    d.nx, d.ny, d.nz = nx, ny, nz
    d.dx, d.dy, d.dz = dx, dy, dz
    keep = []

    def arr(a, dtype, size=None):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dtype).reshape(-1)
        if size is not None and a.size != size:
            raise ValueError(f"expected {size} values, got {a.size}")
        keep.append(a)
        return _ptr(a)

    d.active = arr(active, np.uint8, n)
    d.dt_pde = dt_pde
    d.dt_ode = (1e-10 if ode_adaptive else dt_pde) if dt_ode is None else dt_ode
    d.ode_adaptive = ODE_ADAPTIVE[ode_adaptive]
    d.ode_abs_tol, d.ode_rel_tol = ode_abs_tol, ode_rel_tol
    d.beta, d.cm = beta, cm
    d.model = MODELS[model]
    d.precision = PRECISIONS[precision]
    d.rl_rule = RL_RULES[rl_rule]
    d.initial_state = arr(initial_state, np.float64)
    d.celltype = arr(celltype, np.uint8, n)
    d.current_scale = arr(current_scale, np.float64, _lib.MB_NUM_SCALES * n)
    d.assembly = ASSEMBLIES[assembly]
    d.sigma[0], d.sigma[1], d.sigma[2] = sigma
    d.sigma_l, d.sigma_t = sigma_l, sigma_t
    d.sigma_n = sigma_t if sigma_n is None else sigma_n
    d.fibre_angle_z = arr(fibre_angle_z, np.float64, nz)
    d.sigma_cell = arr(sigma_cell, np.float64, n)
    d.cg_tolerance = cg_tolerance
    d.cg_max_iterations = cg_max_iterations
    d.use_preconditioner = 1 if use_preconditioner else 0
    if len(stims) > _lib.MB_MAX_STIMS:
        raise ValueError("too many stimuli")
    d.num_stims = len(stims)
    for q, s in enumerate(stims):
        t = d.stims[q]
        t.kind = STIM_KINDS[s.kind]
        t.start, t.duration, t.current, t.period = s.start, s.duration, s.current, s.period
        t.x_limit = s.x_limit
        for a in range(3):
            t.min[a] = s.min[a]
            t.max[a] = s.max[a]
        t.cell_mask = arr(s.cell_mask, np.uint8, n)
    d.initial_v = initial_v
    d.track_activation = 1 if track_activation else 0
    d.activation_threshold = activation_threshold
    d.activation_min_interval = activation_min_interval
    if ecg_leads is not None:
        leads = np.ascontiguousarray(np.asarray(ecg_leads, dtype=np.float64).reshape(-1, 3))
        keep.append(leads)
        d.ecg_rate = int(ecg_rate)
        d.ecg_n_leads = leads.shape[0]
        d.ecg_leads = leads.ctypes.data
        d.ecg_sigma_b = float(ecg_sigma_b)
        d.ecg_capacity = int(ecg_capacity)
    return d, keep


class Tissue:
    """One structured-grid tissue solved on the GPU.

    Arrays given per cell are in grid order (index i + nx*(j + ny*k)).
    """

    def __init__(self, nx: int, ny: int, nz: int, dx: float = 100.0, dy: float = 100.0, dz: float = 100.0, *,
                 active: Optional[np.ndarray] = None, dt_pde: float = 0.02, dt_ode: Optional[float] = None,
                 beta: float = 0.14, cm: float = 1.0, model: str = "tt2006", precision: str = "fp64",
                 rl_rule: str = "reference_cpu", assembly: str = "homogeneous",
                 sigma: Sequence[float] = (0.00013, 0.00013, 0.00013), sigma_l: float = 0.0,
                 sigma_t: float = 0.0, sigma_n: Optional[float] = None,
                 fibre_angle_z: Optional[np.ndarray] = None, sigma_cell: Optional[np.ndarray] = None,
                 celltype: Optional[np.ndarray] = None, current_scale: Optional[np.ndarray] = None,
                 initial_state: Optional[np.ndarray] = None, cg_tolerance: float = 1e-16,
                 cg_max_iterations: int = 200, use_preconditioner: bool = True,
                 stims: Sequence[Stim] = (), initial_v: float = float("nan"), track_activation: bool = False,
                 activation_threshold: float = -30.0, activation_min_interval: float = 10.0,
                 ecg_leads: Optional[Sequence[Sequence[float]]] = None, ecg_rate: int = 1, ecg_sigma_b: float = 1.0,
                 ecg_capacity: int = 100000, ode_adaptive: Optional[str] = None, ode_abs_tol: float = 1e-5,
                 ode_rel_tol: float = 1e-5):
        self.shape = (nz, ny, nx)
        self.n = nx * ny * nz
        d, keep = build_desc(nx, ny, nz, dx, dy, dz, active=active, dt_pde=dt_pde, dt_ode=dt_ode, beta=beta,
                             cm=cm, model=model, precision=precision, rl_rule=rl_rule, assembly=assembly,
                             sigma=sigma, sigma_l=sigma_l, sigma_t=sigma_t, sigma_n=sigma_n,
                             fibre_angle_z=fibre_angle_z, sigma_cell=sigma_cell, celltype=celltype,
                             current_scale=current_scale, initial_state=initial_state,
                             cg_tolerance=cg_tolerance, cg_max_iterations=cg_max_iterations,
                             use_preconditioner=use_preconditioner, stims=stims, initial_v=initial_v,
                             track_activation=track_activation, activation_threshold=activation_threshold,
                             activation_min_interval=activation_min_interval, ecg_leads=ecg_leads,
                             ecg_rate=ecg_rate, ecg_sigma_b=ecg_sigma_b, ecg_capacity=ecg_capacity,
                             ode_adaptive=ode_adaptive, ode_abs_tol=ode_abs_tol, ode_rel_tol=ode_rel_tol)
        self.model = model
        self.precision = precision
        self._n_leads = 0 if ecg_leads is None else int(np.asarray(ecg_leads).reshape(-1, 3).shape[0])
        self.active = None if active is None else np.asarray(active, dtype=bool).reshape(-1).copy()
        h = C.c_void_p()
        check(lib.mb_monodomain_create(C.byref(h), C.byref(d)))
        self._h = h
        del keep

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib.mb_monodomain_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- whole steps --------------------------------------------------------
    def step(self, n: int = 1):
        check(lib.mb_monodomain_step(self._h, int(n)))

    def sync(self):
        check(lib.mb_monodomain_sync(self._h))

    def step_host(self, stim: Optional[np.ndarray] = None, v_out: Optional[np.ndarray] = None):
        """One loop step through host buffers (the reference GPU plugins' copies)."""
        check(lib.mb_monodomain_step_host(self._h, _ptr(stim), _ptr(v_out)))

    # -- split API, reference names ----------------------------------------
    def solve_all_volumes_odes(self):
        check(lib.mb_solve_all_volumes_odes(self._h))

    def update_monodomain_default(self):
        check(lib.mb_update_monodomain_default(self._h))

    def conjugate_gradient(self):
        its, err = C.c_uint32(), C.c_double()
        check(lib.mb_conjugate_gradient(self._h, C.byref(its), C.byref(err)))
        return its.value, err.value

    def advance_time(self):
        check(lib.mb_advance_time(self._h))

    # -- state ----------------------------------------------------------------
    def v(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(lib.mb_monodomain_get_v(self._h, _ptr(out)))
        return out

    def set_v(self, v: np.ndarray):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        check(lib.mb_monodomain_set_v(self._h, _ptr(v)))

    def checkpoint(self) -> bytes:
        """The loop state as bytes (mb_monodomain_checkpoint)."""
        n = C.c_size_t()
        check(lib.mb_monodomain_checkpoint_bytes(self._h, C.byref(n)))
        buf = (C.c_char * n.value)()
        check(lib.mb_monodomain_checkpoint(self._h, buf, n.value))
        return bytes(buf)

    def restore(self, state: bytes):
        """Restores a state made by checkpoint() on a tissue of the same kind."""
        buf = C.create_string_buffer(state, len(state))
        check(lib.mb_monodomain_restore(self._h, buf, len(state)))

    def save_state(self, directory: str, gpu_layout: bool = False):
        """The loop state in the three files of the reference's
        save_simulation_state (grid, monodomain solver, ODE solver), which
        the reference's restore_simulation_state reads back."""
        check(lib.mb_monodomain_save_state(self._h, directory.encode(), 1 if gpu_layout else 0))

    def restore_state(self, directory: str):
        """V, the ODE state and the loop clock from the reference's
        save_simulation_state files (written by the reference or by
        save_state) for this tissue's mesh."""
        check(lib.mb_monodomain_restore_state(self._h, directory.encode()))

    def save_v(self, path: str, binary: bool = False):
        """V of the active cells in the reference's save_as_text_or_binary format."""
        check(lib.mb_monodomain_save_v(self._h, path.encode(), 1 if binary else 0))

    def ecg(self):
        """Pseudo-bidomain ECG records taken so far (needs ecg_leads): the
        loop time of each record (ms) and the leads' values, one row per
        record (the columns of the reference's ecg.txt)."""
        n = C.c_int64()
        check(lib.mb_monodomain_get_ecg(self._h, 0, 0, None, None, C.byref(n)))
        t = np.empty(n.value, dtype=np.float64)
        nl = self._n_leads
        vals = np.empty((n.value, nl), dtype=np.float64)
        if n.value:
            check(lib.mb_monodomain_get_ecg(self._h, 0, n.value, _ptr(t), _ptr(vals), C.byref(n)))
        return t, vals

    def activation(self) -> dict:
        """Activation times tracked on the device (needs track_activation):
        first / last activation time and APD90 of the latest beat in ms (-1
        where there is none), and the number of activations, per grid cell."""
        out = {k: np.empty(self.n, dtype=np.float32) for k in ("first", "last", "apd90")}
        out["count"] = np.empty(self.n, dtype=np.int32)
        check(lib.mb_monodomain_get_activation(self._h, _ptr(out["first"]), _ptr(out["last"]), _ptr(out["apd90"]),
                                               _ptr(out["count"])))
        return out

    def info(self):
        count, t, na, neq = C.c_int64(), C.c_double(), C.c_uint32(), C.c_int()
        check(lib.mb_monodomain_info(self._h, C.byref(count), C.byref(t), C.byref(na), C.byref(neq)))
        return {"count": count.value, "cur_time": t.value, "n_active": na.value, "neq": neq.value}

    def state(self) -> np.ndarray:
        inf = self.info()
        out = np.empty((inf["neq"], inf["n_active"]), dtype=np.float64)
        check(lib.mb_monodomain_get_state(self._h, _ptr(out)))
        return out

    def step_stats(self, first: int, n: int) -> np.ndarray:
        buf = (MbStepStats * n)()
        check(lib.mb_monodomain_step_stats(self._h, first, n, buf))
        return np.array([(s.cg_iterations, s.refinements, s.cg_error) for s in buf],
                        dtype=[("its", "i4"), ("refinements", "i4"), ("error", "f8")])

    def device_v(self):
        p, s = C.c_void_p(), C.c_void_p()
        check(lib.mb_monodomain_device_v(self._h, C.byref(p), C.byref(s)))
        return p.value, s.value

    def time_steps(self, n: int) -> float:
        """Device milliseconds of n whole steps (CUDA events on the tissue's stream)."""
        ms = C.c_double()
        check(lib.mb_monodomain_time_steps(self._h, int(n), C.byref(ms)))
        return ms.value

    def time_steps_host(self, n: int, stim_ptr, v_ptr) -> float:
        """Device milliseconds of n steps through host buffers (raw pointers, e.g. pinned memory)."""
        ms = C.c_double()
        check(lib.mb_monodomain_time_steps_host(self._h, int(n), stim_ptr, v_ptr, C.byref(ms)))
        return ms.value

    def time_steps_host_async(self, n: int, stim0: int, stim1: int, v0: int, v1: int) -> float:
        """Device milliseconds of n pipelined host-buffer steps alternating the
        buffer pairs (stim0, v0) and (stim1, v1) (raw addresses of pinned memory)."""
        ms = C.c_double()
        check(lib.mb_monodomain_time_steps_host_async(self._h, int(n), C.c_void_p(stim0), C.c_void_p(stim1),
                                                      C.c_void_p(v0), C.c_void_p(v1), C.byref(ms)))
        return ms.value

    def tuning(self):
        v, b, pc = C.c_int(), C.c_int(), C.c_int()
        check(lib.mb_monodomain_tuning(self._h, C.byref(v), C.byref(b), C.byref(pc)))
        return {"ode_variant": v.value, "cg_blocks": b.value, "cg_kernel": pc.value}

    def profile(self, n: int):
        a, b, c, it = C.c_double(), C.c_double(), C.c_double(), C.c_int()
        check(lib.mb_monodomain_profile_steps(self._h, n, C.byref(a), C.byref(b), C.byref(c), C.byref(it)))
        return {"ode_ms": a.value, "cg_ms": b.value, "step_ms": c.value, "cg_iterations": it.value}


def reference_cell_order(nx: int, ny: int, nz: int, active: Optional[np.ndarray] = None):
    """The reference's numbering of a cuboid's active cells (grid indices in
    its octree's Hilbert order) and the number of leaves of that octree."""
    a = None if active is None else np.ascontiguousarray(active, dtype=np.uint8).reshape(-1)
    n_act, n_leaves = C.c_int64(), C.c_int64()
    check(lib.mb_reference_cell_order(nx, ny, nz, _ptr(a), None, C.byref(n_act), C.byref(n_leaves)))
    order = np.empty(n_act.value, dtype=np.int64)
    check(lib.mb_reference_cell_order(nx, ny, nz, _ptr(a), _ptr(order), C.byref(n_act), C.byref(n_leaves)))
    return order, n_leaves.value


def cg_launch_shapes() -> int:
    """Number of launch shapes of the flat persistent CG (MB_CG_VARIANT values
    0..n-1; n selects the tiled kernel, n + 1 the resident one)."""
    n = C.c_int()
    check(lib.mb_cg_launch_shapes(C.byref(n)))
    return n.value


class OdeSolver:
    """GPU cell-model library for independent cells (set_model_initial_conditions_gpu /
    solve_model_odes_gpu, ode_solver.h:37-47)."""

    def __init__(self, model: str, num_cells: int, dt: float, num_steps: int = 1, precision: str = "fp64",
                 rl_rule: str = "reference_cpu"):
        h = C.c_void_p()
        check(lib.mb_ode_create(C.byref(h), MODELS[model], PRECISIONS[precision], RL_RULES[rl_rule],
                                num_cells, dt, num_steps))
        self._h = h
        self.num_cells = num_cells
        self.neq, self.initial_v = init_cell_model_data(model)
        self.pitch = None

    def set_model_initial_conditions_gpu(self, initial_state: Optional[np.ndarray] = None,
                                         celltype: Optional[np.ndarray] = None) -> int:
        ist = None if initial_state is None else np.ascontiguousarray(initial_state, dtype=np.float64)
        ct = None if celltype is None else np.ascontiguousarray(celltype, dtype=np.uint8)
        pitch = C.c_size_t()
        check(lib.mb_set_model_initial_conditions_gpu(self._h, _ptr(ist), _ptr(ct), C.byref(pitch)))
        self.pitch = pitch.value
        return pitch.value

    def solve_model_odes_gpu(self, current_t: float, stim_currents: Optional[np.ndarray] = None):
        st = None if stim_currents is None else np.ascontiguousarray(stim_currents, dtype=np.float64)
        check(lib.mb_solve_model_odes_gpu(self._h, current_t, _ptr(st)))

    def state(self) -> np.ndarray:
        out = np.empty((self.neq, self.num_cells), dtype=np.float64)
        check(lib.mb_ode_get_state(self._h, _ptr(out)))
        return out

    def set_state(self, s: np.ndarray):
        s = np.ascontiguousarray(s, dtype=np.float64)
        check(lib.mb_ode_set_state(self._h, _ptr(s)))

    def close(self):
        if getattr(self, "_h", None):
            lib.mb_ode_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def csr_conjugate_gradient(row_ptr, col, val, b, x0=None, tolerance=1e-16, max_iterations=200,
                           use_preconditioner=True):
    """Jacobi-PCG on a general CSR matrix (the reference's file-loaded solver test)."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    n = b.size
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    its, err = C.c_uint32(), C.c_double()
    check(lib.mb_csr_conjugate_gradient(n, _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(b), _ptr(x), tolerance,
                                        max_iterations, 1 if use_preconditioner else 0, C.byref(its),
                                        C.byref(err)))
    return x, its.value, err.value

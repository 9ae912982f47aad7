"""ctypes front end of the CPU oracle (oracle/_build/liboracle.so) -- TEST
INFRASTRUCTURE ONLY.

Used by the tests, the smoke check and bench.py's CPU-baseline leg to check
and time against; the product never imports it.  The tissue arguments are
the product's (monoalg3d_c_b200.monodomain.build_desc), so a test hands the
same description to the GPU tissue and to the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def load() -> C.CDLL:
    """Loads the oracle library, building it with make if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    lib = C.CDLL(LIB_PATH)
    vp, i32, u32p, dp = C.c_void_p, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_double)
    lib.orc_create.argtypes = [C.POINTER(vp), vp]
    lib.orc_step.argtypes = [vp, C.c_int]
    lib.orc_get_v.argtypes = [vp, vp]
    lib.orc_get_state.argtypes = [vp, C.c_int, vp]
    lib.orc_last_cg.argtypes = [vp, u32p, dp]
    lib.orc_time.argtypes = [vp]
    lib.orc_time.restype = C.c_double
    lib.orc_active_cells.argtypes = [vp]
    lib.orc_active_cells.restype = i32
    lib.orc_destroy.argtypes = [vp]
    lib.orc_loop_steps.argtypes = [C.c_double, C.c_double]
    lib.orc_tt2006_initial_state.argtypes = [vp]
    lib.orc_tt2006_step.argtypes = [vp, C.c_double, C.c_double, vp]
    lib.orc_torord_initial_state.argtypes = [C.c_int, vp]
    lib.orc_torord_step.argtypes = [vp, C.c_double, C.c_double, C.c_int, C.c_int, vp]
    lib.orc_assemble.argtypes = [vp, vp, vp]
    lib.orc_csr_free.argtypes = [vp]
    lib.orc_pcg.argtypes = [vp, vp, vp, C.c_double, C.c_int, C.c_int, u32p, dp]
    lib.orc_tangent_misfit.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, dp, dp]
    _lib = lib
    return lib


class Csr(C.Structure):
    _fields_ = [("n", C.c_int32), ("row_ptr", C.POINTER(C.c_int32)), ("col", C.POINTER(C.c_int32)),
                ("val", C.POINTER(C.c_double))]


def _p(a: Optional[np.ndarray]):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _desc(nx, ny, nz, **kw):
    from monoalg3d_c_b200.monodomain import build_desc
    return build_desc(nx, ny, nz, **kw)


class Sim:
    """The reference time loop on the CPU for a tissue described with the
    product's arguments (precision is ignored: the oracle is FP64)."""

    def __init__(self, nx: int, ny: int, nz: int, **kw):
        lib = load()
        kw = dict(kw)
        kw.pop("precision", None)
        self.n = nx * ny * nz
        d, keep = _desc(nx, ny, nz, **kw)
        self._keep = (d, keep)            # arrays the description points to
        h = C.c_void_p()
        rc = lib.orc_create(C.byref(h), C.byref(d))
        if rc != 0:
            raise RuntimeError(f"orc_create failed ({rc})")
        self._h = h
        self.model = kw.get("model", "tt2006")

    def step(self, n: int = 1) -> int:
        return load().orc_step(self._h, int(n))

    def v(self) -> np.ndarray:
        out = np.empty(self.n)
        load().orc_get_v(self._h, _p(out))
        return out

    def state(self, var: int) -> np.ndarray:
        out = np.empty(load().orc_active_cells(self._h))
        load().orc_get_state(self._h, int(var), _p(out))
        return out

    def last_cg(self):
        its, err = C.c_uint32(), C.c_double()
        load().orc_last_cg(self._h, C.byref(its), C.byref(err))
        return its.value, err.value

    @property
    def time(self) -> float:
        return load().orc_time(self._h)

    def close(self):
        if getattr(self, "_h", None):
            load().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def assemble(nx: int, ny: int, nz: int, **kw):
    """(row_ptr, col, val, cells) of the tissue's matrix alpha I + K over the
    active cells in grid order; cells = grid index of each row."""
    lib = load()
    d, keep = _desc(nx, ny, nz, **kw)
    A = Csr()
    cells = np.empty(nx * ny * nz, dtype=np.int32)
    rc = lib.orc_assemble(C.byref(d), C.byref(A), _p(cells))
    if rc != 0:
        raise RuntimeError(f"orc_assemble failed ({rc})")
    n = A.n
    rp = np.ctypeslib.as_array(A.row_ptr, shape=(n + 1,)).copy()
    nnz = int(rp[-1])
    col = np.ctypeslib.as_array(A.col, shape=(max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(A.val, shape=(max(nnz, 1),))[:nnz].copy()
    lib.orc_csr_free(C.byref(A))
    return rp, col, val, cells[:n].copy()


def pcg(row_ptr, col, val, b, x0, tol=1e-16, max_its=200, use_preconditioner=True):
    """cpu_conjugate_gradient on a CSR matrix (diagonal first in each row)."""
    lib = load()
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vl = np.ascontiguousarray(val, dtype=np.float64)
    A = Csr(int(rp.size - 1), rp.ctypes.data_as(C.POINTER(C.c_int32)), cl.ctypes.data_as(C.POINTER(C.c_int32)),
            vl.ctypes.data_as(C.POINTER(C.c_double)))
    bb = np.ascontiguousarray(b, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    its, err = C.c_uint32(), C.c_double()
    lib.orc_pcg(C.byref(A), _p(bb), _p(x), tol, int(max_its), 1 if use_preconditioner else 0, C.byref(its),
                C.byref(err))
    return x, its.value, err.value


def tangent_misfit(nx: int, ny: int, nz: int, steps: int, sample_every: int, sensors, target,
                   dsigma: Optional[np.ndarray] = None, dgkr: Optional[np.ndarray] = None, **kw):
    """The loop's L2 misfit 1/2 sum (V at the sensors after every sample_every
    steps - target)^2 and its exact directional derivative along (dsigma,
    dgkr) (per grid cell), from the tangent-linear loop (tangent.cc).
    Returns (loss, dloss)."""
    lib = load()
    kw = dict(kw)
    kw.pop("precision", None)
    d, keep = _desc(nx, ny, nz, **kw)
    sens = np.ascontiguousarray(sensors, dtype=np.int64)
    tgt = np.ascontiguousarray(target, dtype=np.float64)
    ds = None if dsigma is None else np.ascontiguousarray(dsigma, dtype=np.float64)
    dg = None if dgkr is None else np.ascontiguousarray(dgkr, dtype=np.float64)
    loss, dloss = C.c_double(), C.c_double()
    rc = lib.orc_tangent_misfit(C.byref(d), int(steps), int(sample_every), int(sens.size), _p(sens), _p(tgt),
                                _p(ds), _p(dg), C.byref(loss), C.byref(dloss))
    del keep
    if rc != 0:
        raise RuntimeError(f"orc_tangent_misfit failed ({rc})")
    return loss.value, dloss.value


def tt2006_initial_state() -> np.ndarray:
    out = np.empty(19)
    load().orc_tt2006_initial_state(_p(out))
    return out


def torord_initial_state(celltype: int = 0) -> np.ndarray:
    out = np.empty(43)
    load().orc_torord_initial_state(int(celltype), _p(out))
    return out


def loop_steps(final_time: float, dt: float) -> int:
    return load().orc_loop_steps(final_time, dt)


def pseudo_bidomain_ecg(v: np.ndarray, nx: int, ny: int, nz: int, leads, sigma_b: float,
                        dx: float = 100.0, dy: float = 100.0, dz: float = 100.0,
                        active: Optional[np.ndarray] = None) -> np.ndarray:
    """Pseudo-bidomain ECG of the grid-order V at the given electrodes, as
    ecg_library/ecg.c computes it on a cuboid mesh:
      - assembly_divergent / fill_element (ecg.c:36-43, 149-172): per active
        cell, each face neighbour that is an active cell inside the domain
        gets value_ecg = -m and the diagonal +m, with m = dx dy / dz for
        every face direction;
      - pseudo_bidomain_cpu (ecg.c:264-307): beta_im = sum(value_ecg v) / vol,
        lead = -(1 / (4 pi sigma_b)) sum_cells beta_im / |x_cell - lead| vol,
        cell centres at ((i + 1/2) dx, (j + 1/2) dy, (k + 1/2) dz).
    Test infrastructure: the checker of the device ECG."""
    n = nx * ny * nz
    act = np.ones(n, bool) if active is None else np.asarray(active).astype(bool)
    V = np.asarray(v, float).reshape(nz, ny, nx)
    A = act.reshape(nz, ny, nx)
    m = (dx * dy) / dz
    lap = np.zeros_like(V)
    for axis in range(3):
        for shift in (1, -1):
            nb = np.roll(V, shift, axis=axis)
            na = np.roll(A, shift, axis=axis)
            edge = [slice(None)] * 3
            edge[axis] = 0 if shift == 1 else -1
            ok = A & na
            ok[tuple(edge)] = False
            lap += np.where(ok, m * (V - np.where(ok, nb, 0.0)), 0.0)
    vol = dx * dy * dz
    beta = np.where(A, lap / vol, 0.0)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cx, cy, cz = (i + 0.5) * dx, (j + 0.5) * dy, (k + 0.5) * dz
    scale = 1.0 / (4.0 * np.pi * sigma_b)
    out = []
    for (ex, ey, ez) in leads:
        dist = np.sqrt((ex - cx) ** 2 + (ey - cy) ** 2 + (ez - cz) ** 2)
        out.append(-scale * np.sum(np.where(A, beta / dist * vol, 0.0)))
    return np.array(out)

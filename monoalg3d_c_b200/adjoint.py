"""Gradients through the monodomain loop (mb_adjoint_*), and the
torch.autograd.Function that exposes them.

``Adjoint`` runs the loop on the GPU from the tissue's initial state with a
given per-cell conductivity and gKr scaling, returns V sampled at sensor
cells, and maps a gradient of those samples back to gradients with respect to
the conductivity and the gKr scaling (discrete adjoint, checkpoints every
``checkpoint_every`` steps, states in between recomputed).

``traces(sigma, gkr, adjoint)`` is the autograd entry: forward gives the
samples as a tensor, backward the two gradients.  The adjoint object keeps the
checkpoints of its latest forward run, so each backward must follow its own
forward before the next forward on the same object.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from ._lib import MB_NUM_SCALES, check, lib
from .monodomain import _ptr, build_desc


class Adjoint:
    """Loop + adjoint on an nx x ny x nz grid with per-cell conductivity.

    sigma_cell: conductivity per cell (mS/um, grid order); gkr: gKr scaling per
    cell; sensors: grid indices; samples after every ``sample_every`` steps.
    Other keywords go to the tissue description (dt_pde, stims, cg_tolerance,
    ...); the model is ten Tusscher 2006.  precision "mixed" runs the forward
    in the mixed form (FP32 cell model and CG recurrences) and its adjoint
    with the cell model's Jacobian in FP32, every adjoint vector and gradient
    accumulated in FP64.
    """

    def __init__(self, nx: int, ny: int, nz: int, sigma_cell: np.ndarray, gkr: np.ndarray, sensors: Sequence[int],
                 nsteps: int, sample_every: int, checkpoint_every: int = 50, precision: str = "fp64", **kw):
        self.n = nx * ny * nz
        self.ns = len(sensors)
        self.nsamples = nsteps // sample_every
        scale = self.scales(gkr)
        d, keep = build_desc(nx, ny, nz, model="tt2006", precision=precision, assembly="per_cell",
                             sigma_cell=np.asarray(sigma_cell, dtype=np.float64), current_scale=scale, **kw)
        sens = np.ascontiguousarray(sensors, dtype=np.int64)
        h = C.c_void_p()
        check(lib.mb_adjoint_create(C.byref(h), C.byref(d), int(nsteps), int(checkpoint_every), self.ns,
                                    _ptr(sens), int(sample_every)))
        self._h = h
        del keep

    def scales(self, gkr: np.ndarray) -> np.ndarray:
        s = np.ones((MB_NUM_SCALES, self.n), dtype=np.float64)
        s[1] = np.asarray(gkr, dtype=np.float64).reshape(-1)
        return s

    def forward(self, sigma_cell: Optional[np.ndarray] = None, gkr: Optional[np.ndarray] = None) -> np.ndarray:
        sig = None if sigma_cell is None else np.ascontiguousarray(sigma_cell, dtype=np.float64).reshape(-1)
        sc = None if gkr is None else self.scales(gkr)
        out = np.empty((self.nsamples, self.ns), dtype=np.float64)
        check(lib.mb_adjoint_forward(self._h, _ptr(sig), _ptr(sc), _ptr(out)))
        return out

    def backward(self, dtraces: np.ndarray):
        g = np.ascontiguousarray(dtraces, dtype=np.float64).reshape(self.nsamples, self.ns)
        gs = np.empty(self.n, dtype=np.float64)
        gk = np.empty(self.n, dtype=np.float64)
        check(lib.mb_adjoint_backward(self._h, _ptr(g), _ptr(gs), _ptr(gk)))
        return gs, gk

    def close(self):
        if getattr(self, "_h", None):
            lib.mb_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _function():
    import torch

    class MonodomainTraces(torch.autograd.Function):
        """forward(sigma, gkr) -> V samples at the sensors; backward -> dL/dsigma, dL/dgkr."""

        @staticmethod
        def forward(ctx, sigma, gkr, adj):
            tr = adj.forward(sigma.detach().cpu().double().numpy(), gkr.detach().cpu().double().numpy())
            ctx.adj = adj
            ctx.device = sigma.device
            return torch.from_numpy(tr).to(sigma.device)

        @staticmethod
        def backward(ctx, g):
            gs, gk = ctx.adj.backward(g.detach().cpu().double().numpy())
            return torch.from_numpy(gs).to(ctx.device), torch.from_numpy(gk).to(ctx.device), None

    return MonodomainTraces


_FN = None


def traces(sigma, gkr, adj: Adjoint):
    """Autograd entry: V samples (samples x sensors) as a function of the
    per-cell conductivity and gKr scaling (float64 tensors of the grid size)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(sigma, gkr, adj)

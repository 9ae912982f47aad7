"""Batches of independent tissues solved as one (mb_batch_pack).

The tissues -- 2-D sheets nx x ny, cables with ny = 1 -- are packed into one
atlas grid with removed cells between them; the atlas is an ordinary Tissue,
so one ODE launch, one persistent CG launch and one graph replay per step
advance the whole batch.  Per-tissue conductance scalings and stimulus
regions become per-cell arrays.  Results come back per tissue.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from ._lib import MB_NUM_SCALES, check, lib
from .monodomain import Stim, Tissue


def pack(sizes: Sequence[Tuple[int, int]]):
    """(atlas_nx, atlas_ny, x0, y0) for tissues of sizes (nx, ny)."""
    n = len(sizes)
    nx = np.array([s[0] for s in sizes], dtype=np.int32)
    ny = np.array([s[1] for s in sizes], dtype=np.int32)
    x0 = np.empty(n, dtype=np.int32)
    y0 = np.empty(n, dtype=np.int32)
    W, H = C.c_int32(), C.c_int32()
    check(lib.mb_batch_pack(n, C.c_void_p(nx.ctypes.data), C.c_void_p(ny.ctypes.data), C.byref(W), C.byref(H),
                            C.c_void_p(x0.ctypes.data), C.c_void_p(y0.ctypes.data)))
    return W.value, H.value, x0, y0


def atlas(sizes: Sequence[Tuple[int, int]], scales: Optional[np.ndarray], stim: Stim, dx: float = 100.0):
    """(atlas_nx, atlas_ny, x0, y0, Tissue keywords) of the atlas holding the
    tissues: the active mask, per-cell scalings and the stimulus mask."""
    sizes = [(int(a), int(b)) for a, b in sizes]
    W, H, x0, y0 = pack(sizes)
    n = W * H
    active = np.zeros((H, W), dtype=np.uint8)
    stim_mask = np.zeros((H, W), dtype=np.uint8)
    scale = np.ones((MB_NUM_SCALES, H, W), dtype=np.float64)
    for q, (nx, ny) in enumerate(sizes):
        sl = (slice(y0[q], y0[q] + ny), slice(x0[q], x0[q] + nx))
        active[sl] = 1
        cx = (np.arange(nx) + 0.5) * dx
        stim_mask[sl] = (cx < stim.x_limit)[None, :]
        if scales is not None:
            scale[(slice(None),) + sl] = np.asarray(scales[q], dtype=np.float64)[:, None, None]
    stims = [Stim(kind="cell_mask", start=stim.start, duration=stim.duration, current=stim.current,
                  period=stim.period, cell_mask=stim_mask.reshape(-1))]
    kw = dict(active=active.reshape(-1), stims=stims,
              current_scale=None if scales is None else scale.reshape(MB_NUM_SCALES, n))
    return W, H, x0, y0, kw


class Batch:
    """Independent 2-D tissues (sheets, cables) solved in one atlas tissue.

    sizes:  (nx, ny) per tissue
    scales: (n, 5) conductance scalings per tissue (gNa, gKr, gKs, gCaL, gK1)
    stim:   start / duration / current / period of the stimulus applied, in
            every tissue, to the cells whose centre x is below stim.x_limit (um)
    Every other keyword goes to Tissue (model, precision, sigma, dt, ...).
    """

    def __init__(self, sizes: Sequence[Tuple[int, int]], scales: Optional[np.ndarray] = None,
                 stim: Stim = Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=100.0),
                 dx: float = 100.0, **kw):
        self.sizes = [(int(a), int(b)) for a, b in sizes]
        W, H, x0, y0, akw = atlas(self.sizes, scales, stim, dx)
        self.atlas = (W, H)
        self.x0, self.y0 = x0, y0
        self.active_cells = int(akw["active"].sum())
        akw.update(kw)
        self.tissue = Tissue(W, H, 1, dx, dx, dx, **akw)

    def split(self, grid: np.ndarray) -> List[np.ndarray]:
        """Per-tissue (ny, nx) views of an atlas array in grid order."""
        W, H = self.atlas
        g = np.asarray(grid).reshape(H, W)
        return [g[self.y0[q]:self.y0[q] + ny, self.x0[q]:self.x0[q] + nx] for q, (nx, ny) in enumerate(self.sizes)]

    def step(self, n: int = 1):
        self.tissue.step(n)

    def v(self) -> List[np.ndarray]:
        return self.split(self.tissue.v())

    def activation(self) -> List[dict]:
        a = self.tissue.activation()
        parts = {k: self.split(v) for k, v in a.items()}
        return [{k: parts[k][q] for k in parts} for q in range(len(self.sizes))]

    def close(self):
        self.tissue.close()

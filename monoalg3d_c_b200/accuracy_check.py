"""Error of the mixed-precision form against the plain FP64 path on one of the
bench workloads: the same tissue run in both precisions for the same time,
with activation tracked on the device (threshold -30 mV).  Prints one JSON
line with

  - V at the end: RMS and max |difference| in mV over the active cells;
  - first activation time: max and RMS |difference| in ms over the cells
    activated in both runs, and the number of cells activated in only one;
  - latest activation time, over the cells with the same number of
    activations in both runs (every beat of a re-entrant run is compared
    through it and the first);
  - APD90 of the latest beat: max and RMS |difference| in ms over the cells
    whose beat completed in both runs, the number of them above 0.5 ms, and
    the same over the cells with the same number of activations in both runs
    (a cell re-excited in one run only measures a different beat).

With --trace, V of a set of watched cells is also sampled every 1 ms in both
runs (gathered on the device): a band of cells along the boundary of the
second stimulus' box (where cells are caught at the edge of refractoriness)
and a random sample.  Every cell whose APD90 differs by more than 0.5 ms or
whose activation count differs is then classified from its traces where it
was watched: whether V re-crosses its 90 % repolarisation level after the
first downward crossing (a bump on a flat late repolarisation, which makes
the first-crossing time jump), and whether an extra activation follows the
second stimulus.

    python -m monoalg3d_c_b200.accuracy_check [--config 1] [--ms 400] [--scale 1.0] [--trace]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


class _DeviceV:
    """V of a tissue in device memory, as a zero-copy CUDA array."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


def _run(wl, precision: str, steps: int, watch=None, every: int = 50):
    t = wl.tissue(precision=precision, track_activation=True)
    traces = None
    t0 = time.perf_counter()
    if watch is None:
        t.step(steps)
        t.sync()
    else:
        import torch
        ptr, _ = t.device_v()
        vdev = torch.as_tensor(_DeviceV(ptr, wl.n), device="cuda")
        idx = torch.as_tensor(watch, device="cuda")
        nsamp = steps // every
        traces = np.empty((len(watch), nsamp), dtype=np.float32)
        for k in range(nsamp):
            t.step(every)
            t.sync()
            traces[:, k] = vdev[idx].float().cpu().numpy()
        t.step(steps - nsamp * every)
        t.sync()
    secs = time.perf_counter() - t0
    v = t.v()
    act = t.activation()
    t.close()
    return v, act, secs, traces


def _stats(d: np.ndarray):
    if d.size == 0:
        return {"max": None, "rms": None, "cells": 0}
    return {"max": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d))), "cells": int(d.size),
            "cells_over_0.5": int(np.count_nonzero(np.abs(d) > 0.5))}     # in the block's unit (mV or ms)


def _watch_cells(wl, s2, seed: int = 7):
    """Grid indices of a band two cells wide on each side of the boundary of
    the second stimulus' box (x, y <= its max), every z, plus 20000 random
    cells."""
    nx, ny, nz = wl.nx, wl.ny, wl.nz
    dx = wl.kwargs.get("dx", 100.0)
    ix = int(np.floor(s2.max[0] / dx - 0.5))  # last stimulated column: centre (i + 1/2) dx <= max
    iy = int(np.floor(s2.max[1] / dx - 0.5))
    i = np.arange(nx)[None, None, :]
    j = np.arange(ny)[None, :, None]
    band = (((np.abs(i - ix - 0.5) <= 2) & (j <= iy + 2)) | ((np.abs(j - iy - 0.5) <= 2) & (i <= ix + 2)))
    band = np.broadcast_to(band, (nz, ny, nx)).reshape(-1)
    sel = np.nonzero(band)[0]
    rnd = np.random.default_rng(seed).choice(wl.n, size=min(20000, wl.n), replace=False)
    return np.unique(np.concatenate([sel, rnd])).astype(np.int64), ix, iy


def _diagnose(wl, a_mx, a_64, tr_mx, tr_64, watch, ix, iy, s2_start, every_ms=1.0):
    """Classifies the outlier cells from their traces (see the module text)."""
    same = a_mx["count"] == a_64["count"]
    apd = (a_mx["apd90"] > 0) & (a_64["apd90"] > 0)
    out_apd = np.nonzero(same & apd & (np.abs(a_mx["apd90"].astype(np.float64) - a_64["apd90"]) > 0.5))[0]
    out_cnt = np.nonzero(~same)[0]
    pos = {int(g): q for q, g in enumerate(watch)}

    def recross(trace, t_act):
        """Downward crossings of the 90 % level after the activation at t_act."""
        k0 = int(np.ceil(t_act / every_ms))
        seg = trace[k0:].astype(np.float64)
        if seg.size < 3:
            return 0
        pk = seg.max()
        rest = trace[:max(k0, 1)].min()
        v90 = pk - 0.9 * (pk - rest)
        below = seg <= v90
        return int(np.count_nonzero(below[1:] & ~below[:-1]))

    nx, ny = wl.nx, wl.ny
    rows = []
    mech = {"apd_bump_recross": 0, "apd_no_trace": 0, "apd_other": 0, "count_after_s2": 0, "count_no_trace": 0,
            "count_other": 0}
    for g in out_apd:
        q = pos.get(int(g))
        if q is None:
            mech["apd_no_trace"] += 1
            continue
        r1 = recross(tr_mx[q], float(a_mx["last"][g]))
        r2 = recross(tr_64[q], float(a_64["last"][g]))
        mech["apd_bump_recross" if max(r1, r2) > 1 else "apd_other"] += 1
        if len(rows) < 12:
            rows.append(dict(kind="apd90", cell=int(g), i=int(g % nx), j=int((g // nx) % ny), k=int(g // (nx * ny)),
                             apd_mixed=float(a_mx["apd90"][g]), apd_fp64=float(a_64["apd90"][g]),
                             count=int(a_mx["count"][g]), v90_crossings=[r1, r2]))
    for g in out_cnt:
        q = pos.get(int(g))
        late = max(float(a_mx["last"][g]), float(a_64["last"][g])) >= s2_start
        if q is None:
            mech["count_no_trace"] += 1
        else:
            mech["count_after_s2" if late else "count_other"] += 1
        if len(rows) < 24:
            rows.append(dict(kind="count", cell=int(g), i=int(g % nx), j=int((g // nx) % ny), k=int(g // (nx * ny)),
                             counts=[int(a_mx["count"][g]), int(a_64["count"][g])],
                             last=[float(a_mx["last"][g]), float(a_64["last"][g])], watched=q is not None,
                             s2_box_edge_cells=[ix, iy]))
    return {"apd90_outliers": int(out_apd.size), "count_outliers": int(out_cnt.size), "mechanisms": mech,
            "examples": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 4])
    ap.add_argument("--ms", type=float, default=400.0, help="simulated time")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--trace", action="store_true", help="classify the outliers from 1 ms V traces")
    args = ap.parse_args()
    from . import monodomain, workloads
    wl = workloads.CONFIGS[args.config](args.scale)
    steps = monodomain.loop_steps(args.ms, 0.02)
    watch = s2 = None
    if args.trace:
        stims = wl.kwargs.get("stims", ())
        s2 = next((s for s in stims if s.kind == "x_y_limits"), None)
        if s2 is not None:
            watch, ix, iy = _watch_cells(wl, s2)
    v_mx, a_mx, s_mx, tr_mx = _run(wl, "mixed", steps, watch)
    v_64, a_64, s_64, tr_64 = _run(wl, "fp64", steps, watch)
    ok = np.isfinite(v_64) & np.isfinite(v_mx)
    f_mx, f_64 = a_mx["first"], a_64["first"]
    both = (f_mx >= 0) & (f_64 >= 0)
    one = (f_mx >= 0) != (f_64 >= 0)
    p_mx, p_64 = a_mx["apd90"], a_64["apd90"]
    apd = (p_mx > 0) & (p_64 > 0)
    same_n = a_mx["count"] == a_64["count"]
    l_both = same_n & (a_mx["last"] >= 0) & (a_64["last"] >= 0)
    out = {
        "workload": wl.name, "cells": wl.n, "simulated_ms": args.ms, "steps": steps,
        "seconds": {"mixed": s_mx, "fp64": s_64},
        "v_mv": _stats(v_mx[ok] - v_64[ok]),
        "activation_ms": dict(_stats(f_mx[both].astype(np.float64) - f_64[both].astype(np.float64)),
                              activated_in_one_run_only=int(one.sum())),
        "latest_activation_ms_same_count": _stats(a_mx["last"][l_both].astype(np.float64)
                                                  - a_64["last"][l_both].astype(np.float64)),
        "activations": {"total_mixed": int(a_mx["count"].sum()), "total_fp64": int(a_64["count"].sum()),
                        "cells_with_more_than_one": int(np.count_nonzero(a_64["count"] > 1))},
        "apd90_ms": _stats(p_mx[apd].astype(np.float64) - p_64[apd].astype(np.float64)),
    }
    same = apd & same_n
    out["apd90_ms_same_beat_count"] = dict(_stats(p_mx[same].astype(np.float64) - p_64[same].astype(np.float64)),
                                           activation_count_differs=int(np.count_nonzero(~same_n)))
    if watch is not None:
        out["outliers"] = _diagnose(wl, a_mx, a_64, tr_mx, tr_64, watch, ix, iy, s2.start)
        out["outliers"]["watched_cells"] = int(len(watch))
    print(json.dumps(out))


if __name__ == "__main__":
    main()

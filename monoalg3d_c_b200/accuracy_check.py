"""Error of the mixed-precision form against the plain FP64 path on one of the
bench workloads: the same tissue run in both precisions for the same time,
with activation tracked on the device (threshold -30 mV).  Prints one JSON
line with

  - V at the end: RMS and max |difference| in mV over the active cells;
  - first activation time: max and RMS |difference| in ms over the cells
    activated in both runs, and the number of cells activated in only one;
  - APD90 of the latest beat: max and RMS |difference| in ms over the cells
    whose beat completed in both runs, the number of them above 0.5 ms, and
    the same over the cells with the same number of activations in both runs
    (a cell re-excited in one run only measures a different beat).

    python -m monoalg3d_c_b200.accuracy_check [--config 1] [--ms 400] [--scale 1.0]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def _run(wl, precision: str, steps: int):
    t = wl.tissue(precision=precision, track_activation=True)
    t0 = time.perf_counter()
    t.step(steps)
    t.sync()
    secs = time.perf_counter() - t0
    v = t.v()
    act = t.activation()
    t.close()
    return v, act, secs


def _stats(d: np.ndarray):
    if d.size == 0:
        return {"max": None, "rms": None, "cells": 0}
    return {"max": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d))), "cells": int(d.size),
            "cells_over_0.5": int(np.count_nonzero(np.abs(d) > 0.5))}     # in the block's unit (mV or ms)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 4])
    ap.add_argument("--ms", type=float, default=400.0, help="simulated time")
    ap.add_argument("--scale", type=float, default=1.0)
    args = ap.parse_args()
    from . import workloads
    wl = workloads.CONFIGS[args.config](args.scale)
    steps = int(round(args.ms / 0.02))
    v_mx, a_mx, s_mx = _run(wl, "mixed", steps)
    v_64, a_64, s_64 = _run(wl, "fp64", steps)
    ok = np.isfinite(v_64) & np.isfinite(v_mx)
    f_mx, f_64 = a_mx["first"], a_64["first"]
    both = (f_mx >= 0) & (f_64 >= 0)
    one = (f_mx >= 0) != (f_64 >= 0)
    p_mx, p_64 = a_mx["apd90"], a_64["apd90"]
    apd = (p_mx > 0) & (p_64 > 0)
    out = {
        "workload": wl.name, "cells": wl.n, "simulated_ms": args.ms, "steps": steps,
        "seconds": {"mixed": s_mx, "fp64": s_64},
        "v_mv": _stats(v_mx[ok] - v_64[ok]),
        "activation_ms": dict(_stats(f_mx[both].astype(np.float64) - f_64[both].astype(np.float64)),
                              activated_in_one_run_only=int(one.sum())),
        "apd90_ms": _stats(p_mx[apd].astype(np.float64) - p_64[apd].astype(np.float64)),
    }
    same = apd & (a_mx["count"] == a_64["count"])
    out["apd90_ms_same_beat_count"] = dict(_stats(p_mx[same].astype(np.float64) - p_64[same].astype(np.float64)),
                                           activation_count_differs=int(np.count_nonzero(
                                               a_mx["count"] != a_64["count"])))
    print(json.dumps(out))


if __name__ == "__main__":
    main()

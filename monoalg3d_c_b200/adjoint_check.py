"""The differentiation configuration end to end: the observation traces from
the correlated conductivity field, the gradient of the L2 misfit at uniform
conductivity and gKr scaling 1 by the discrete adjoint, and its check
against central finite differences of the same loop along random directions.
With --precision mixed the loop runs in the mixed form (FP32 cell model and
CG recurrences, FP64 V, concentrations, dot products and gradient
accumulation) and the directional derivatives are also compared with those
of the FP64 adjoint at the same point.  Prints one JSON line (times,
directional derivatives, relative errors).

    python -m monoalg3d_c_b200.adjoint_check [--dirs 32] [--scale 1.0] [--precision mixed]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dirs", type=int, default=32)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--h", type=float, default=None, help="relative step of the sigma differences")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    args = ap.parse_args()
    # FP32 forward: a step large enough that the differences rise above its rounding
    h = args.h if args.h is not None else (1e-4 if args.precision == "fp64" else 1e-2)
    from . import workloads
    from .adjoint import Adjoint
    p = workloads.config3(args.scale)
    nx, ny = p["nx"], p["ny"]
    kw = dict(nsteps=p["nsteps"], sample_every=p["sample_every"], checkpoint_every=p["checkpoint_every"],
              stims=p["stims"], cg_tolerance=1e-24, cg_max_iterations=500)
    adj = Adjoint(nx, ny, 1, p["sigma0"], p["gkr0"], p["sensors"], precision=args.precision, **kw)
    target = adj.forward(p["sigma_true"], p["gkr0"])
    t0 = time.perf_counter()
    tr = adj.forward(p["sigma0"], p["gkr0"])
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    gs, gk = adj.backward(tr - target)
    t_bwd = time.perf_counter() - t0
    loss = lambda t: 0.5 * float(np.sum((t - target) ** 2))  # noqa: E731
    ref = None
    if args.precision == "mixed":
        # the FP64 adjoint at the same point, against the same target
        a64 = Adjoint(nx, ny, 1, p["sigma0"], p["gkr0"], p["sensors"], precision="fp64", **kw)
        t64 = a64.forward(p["sigma0"], p["gkr0"])
        ref = a64.backward(t64 - target)
        a64.close()
    r = np.random.Generator(np.random.Philox(3004))
    errs, rows = [], []
    for q in range(args.dirs):
        d = r.standard_normal(nx * ny)
        if q % 2 == 0:          # conductivity direction, relative
            lp = loss(adj.forward(p["sigma0"] * (1 + h * d), p["gkr0"]))
            lm = loss(adj.forward(p["sigma0"] * (1 - h * d), p["gkr0"]))
            fd = (lp - lm) / (2 * h)
            ad = float(np.sum(gs * p["sigma0"] * d))
            ad64 = None if ref is None else float(np.sum(ref[0] * p["sigma0"] * d))
            kind = "sigma"
        else:                   # gKr direction; the scaling is applied as a float
            kp = np.float32(p["gkr0"] * (1 + 1e-2 * d)).astype(np.float64)
            km = np.float32(p["gkr0"] * (1 - 1e-2 * d)).astype(np.float64)
            fd = (loss(adj.forward(p["sigma0"], kp)) - loss(adj.forward(p["sigma0"], km))) / 2.0
            ad = float(np.sum(gk * (kp - km)) / 2.0)
            ad64 = None if ref is None else float(np.sum(ref[1] * (kp - km)) / 2.0)
            kind = "gkr"
        err = abs(ad - fd) / max(abs(fd), 1e-300)
        errs.append(err)
        row = {"kind": kind, "adjoint": ad, "fd": fd, "rel_err": err}
        if ad64 is not None:
            row["fp64_adjoint"] = ad64
            row["rel_diff_fp64_adjoint"] = abs(ad - ad64) / max(abs(ad64), 1e-300)
        rows.append(row)
    adj.close()
    cells = nx * ny
    extra = {}
    if ref is not None:
        d64 = [r["rel_diff_fp64_adjoint"] for r in rows]
        extra = {"max_rel_diff_fp64_adjoint": max(d64), "median_rel_diff_fp64_adjoint": float(np.median(d64))}
    print(json.dumps({"config": f"sheet {nx}x{ny} TT2006, {p['nsteps']} steps, 64 sensors", "precision": args.precision,
                      "sigma_step": h, **extra,
                      "forward_s": t_fwd, "backward_s": t_bwd,
                      "forward_cell_steps_per_s": cells * p["nsteps"] / t_fwd,
                      "loss": loss(tr), "directions": args.dirs, "max_rel_err": max(errs),
                      "median_rel_err": float(np.median(errs)), "per_direction": rows}))


if __name__ == "__main__":
    main()

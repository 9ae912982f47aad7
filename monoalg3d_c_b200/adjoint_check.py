"""The differentiation configuration end to end: the observation traces from
the correlated conductivity field, the gradient of the L2 misfit at uniform
conductivity and gKr scaling 1 by the discrete adjoint, and its check
against central finite differences of the same loop along random directions.
Prints one JSON line (times, directional derivatives, relative errors).

    python -m monoalg3d_c_b200.adjoint_check [--dirs 32] [--scale 1.0]
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
    ap.add_argument("--h", type=float, default=1e-4)
    args = ap.parse_args()
    from . import workloads
    from .adjoint import Adjoint
    p = workloads.config3(args.scale)
    nx, ny = p["nx"], p["ny"]
    adj = Adjoint(nx, ny, 1, p["sigma0"], p["gkr0"], p["sensors"], nsteps=p["nsteps"],
                  sample_every=p["sample_every"], checkpoint_every=p["checkpoint_every"], stims=p["stims"],
                  cg_tolerance=1e-24, cg_max_iterations=500)
    target = adj.forward(p["sigma_true"], p["gkr0"])
    t0 = time.perf_counter()
    tr = adj.forward(p["sigma0"], p["gkr0"])
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    gs, gk = adj.backward(tr - target)
    t_bwd = time.perf_counter() - t0
    loss = lambda t: 0.5 * float(np.sum((t - target) ** 2))  # noqa: E731
    r = np.random.Generator(np.random.Philox(3004))
    errs, rows = [], []
    for q in range(args.dirs):
        d = r.standard_normal(nx * ny)
        if q % 2 == 0:          # conductivity direction, relative
            lp = loss(adj.forward(p["sigma0"] * (1 + args.h * d), p["gkr0"]))
            lm = loss(adj.forward(p["sigma0"] * (1 - args.h * d), p["gkr0"]))
            fd = (lp - lm) / (2 * args.h)
            ad = float(np.sum(gs * p["sigma0"] * d))
            kind = "sigma"
        else:                   # gKr direction; the scaling is applied as a float
            kp = np.float32(p["gkr0"] * (1 + 1e-2 * d)).astype(np.float64)
            km = np.float32(p["gkr0"] * (1 - 1e-2 * d)).astype(np.float64)
            fd = (loss(adj.forward(p["sigma0"], kp)) - loss(adj.forward(p["sigma0"], km))) / 2.0
            ad = float(np.sum(gk * (kp - km)) / 2.0)
            kind = "gkr"
        err = abs(ad - fd) / max(abs(fd), 1e-300)
        errs.append(err)
        rows.append({"kind": kind, "adjoint": ad, "fd": fd, "rel_err": err})
    adj.close()
    cells = nx * ny
    print(json.dumps({"config": f"sheet {nx}x{ny} TT2006, {p['nsteps']} steps, 64 sensors",
                      "forward_s": t_fwd, "backward_s": t_bwd,
                      "forward_cell_steps_per_s": cells * p["nsteps"] / t_fwd,
                      "loss": loss(tr), "directions": args.dirs, "max_rel_err": max(errs),
                      "median_rel_err": float(np.median(errs)), "per_direction": rows}))


if __name__ == "__main__":
    main()

"""A short run of a benchmark tissue for profilers: creates the tissue of a
configuration at a scale, steps it a few times and prints its tuning and a
per-phase timing.  Launch choices can be forced through the environment the
tissue reads at creation: MB_ODE_VARIANT (cell-model kernel) and
MB_CG_VARIANT (CG form and launch shape: the flat shapes, then the tiled,
resident and z-march kernels, as `Tissue.tuning()` reports them).

    python -m monoalg3d_c_b200.profile_run [--config 4] [--scale 0.72] [--precision mixed] [--steps 5]

Under ncu, the tissue's first solve after creation is its first CG launch
that is not a tuning run (the tuner launches each candidate three times).
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=4, choices=[0, 1, 4])
    ap.add_argument("--scale", type=float, default=0.72)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--steps", type=int, default=5)
    args = ap.parse_args()
    from . import workloads
    wl = {0: workloads.config0, 1: workloads.config1, 4: workloads.config4}[args.config](args.scale)
    t = wl.tissue(precision=args.precision)
    t.step(max(args.steps - 2, 1))
    t.sync()
    prof = t.profile(2)
    print(json.dumps({"precision": args.precision, "tuning": t.tuning(), "profile": prof, "info": t.info()}))
    t.close()


if __name__ == "__main__":
    main()

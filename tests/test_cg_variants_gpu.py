"""Every launch shape of the persistent CG (one cell per thread, U cells per
thread, four-cell groups, each with per-block ranges and interleaved sweeps;
2.5D tiles; for the 27-point operator the z-march kernel's variants, whose
stencil input is staged by TMA) against the CPU oracle on each
operator kind: constant coefficients with removed cells, per-cell
conductivity, and the 27-point rows of fibres rotating through the wall.
The shape the autotuner would pick is forced through MB_CG_VARIANT, which
the tissue reads when it is created.  Bar: V within 1e-8 relative (FP64);
for the mixed-precision solve, whose refinements interleave reductions of
three values with the iteration's one and two, every shape (and the
resident kernel where the operator allows it) within 2e-3 relative of the
FP64 oracle and the same iteration counts as shape 0 within one."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

STEPS = 120
# z-march variants per precision: the mixed table adds three of the fused
# single-reduction iteration
ZMARCH_VARIANTS = {"fp64": 7, "mixed": 10}


def _kernel_id(v: int, nf: int) -> int:
    """The cg_kernel id mb_monodomain_tuning reports for MB_CG_VARIANT=v."""
    if v < nf:
        return v
    return {nf: 100, nf + 1: 200}.get(v, 300 + (v - nf - 2))


def _cases():
    rng = np.random.default_rng(31)
    nx, ny, nz = 24, 12, 5
    n = nx * ny * nz
    return {
        "masked": (nx, ny, nz, dict(active=(rng.random(n) >= 0.2).astype(np.uint8), model="torord",
                                    assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00005)),
        "per_cell": (nx, ny, nz, dict(assembly="per_cell", sigma_cell=0.00013 * np.exp(0.3 * rng.standard_normal(n)),
                                      active=(rng.random(n) >= 0.1).astype(np.uint8))),
        "rotating": (nx, ny, nz, dict(assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00004,
                                      fibre_angle_z=np.deg2rad(np.linspace(60, -60, nz)))),
    }


@pytest.mark.parametrize("case", ["masked", "per_cell", "rotating"])
def test_every_launch_shape_matches_oracle(case):
    from monoalg3d_c_b200 import Stim, Tissue
    nx, ny, nz, kw = _cases()[case]
    stims = [Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)]
    o = oracle.Sim(nx, ny, nz, stims=stims, **kw)
    o.step(STEPS)
    ref = o.v()
    o.close()
    ok = np.isfinite(ref)
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    nf = cg_launch_shapes()
    # flat shapes (two sweep orders), the tiled kernel, and for the 27-point
    # operator the z-march variants (MB_CG_VARIANT nf + 2 + v)
    variants = list(range(nf + 1)) + ([nf + 2 + z for z in range(ZMARCH_VARIANTS["fp64"])]
                                      if case == "rotating" else [])
    old = os.environ.get("MB_CG_VARIANT")
    try:
        for v in variants:
            os.environ["MB_CG_VARIANT"] = str(v)
            t = Tissue(nx, ny, nz, precision="fp64", stims=stims, **kw)
            kernel = t.tuning()["cg_kernel"]
            assert kernel == _kernel_id(v, nf), f"variant {v} not used ({kernel})"
            t.step(STEPS)
            got = t.v()
            t.close()
            err = np.abs(got[ok] - ref[ok])
            assert np.all(err <= 1e-8 * np.abs(ref[ok]) + 1e-9), f"{case} variant {v}: max |dV| {err.max():.3e}"
    finally:
        if old is None:
            os.environ.pop("MB_CG_VARIANT", None)
        else:
            os.environ["MB_CG_VARIANT"] = old


@pytest.mark.parametrize("case", ["masked", "per_cell", "rotating"])
def test_every_launch_shape_mixed(case):
    from monoalg3d_c_b200 import Stim, Tissue
    nx, ny, nz, kw = _cases()[case]
    stims = [Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)]
    o = oracle.Sim(nx, ny, nz, stims=stims, **kw)
    o.step(STEPS)
    ref = o.v()
    o.close()
    ok = np.isfinite(ref)
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    nf = cg_launch_shapes()
    old = os.environ.get("MB_CG_VARIANT")
    its0 = None
    try:
        variants = list(range(nf + 2)) + ([nf + 2 + z for z in range(ZMARCH_VARIANTS["mixed"])]
                                          if case == "rotating" else [])
        for v in variants:                        # flat shapes, tiled, resident, z-march
            os.environ["MB_CG_VARIANT"] = str(v)
            t = Tissue(nx, ny, nz, precision="mixed", stims=stims, **kw)
            kernel = t.tuning()["cg_kernel"]
            if v == nf + 1 and kernel != 200:
                t.close()                         # the resident kernel does not apply to this operator
                continue
            assert kernel == _kernel_id(v, nf), f"variant {v} not used ({kernel})"
            t.step(STEPS)
            got = t.v()
            its = t.step_stats(0, STEPS)["its"]
            t.close()
            if its0 is None:
                its0 = its
            assert np.abs(its - its0).max() <= 1, f"{case} variant {v}: iteration counts differ from shape 0"
            err = np.abs(got[ok] - ref[ok])
            assert np.all(err <= 2e-3 * (np.abs(ref[ok]) + 1.0)), f"{case} variant {v}: max |dV| {err.max():.3e}"
    finally:
        if old is None:
            os.environ.pop("MB_CG_VARIANT", None)
        else:
            os.environ["MB_CG_VARIANT"] = old

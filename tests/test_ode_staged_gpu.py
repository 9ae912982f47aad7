"""The staged persistent ODE kernels (ODE variants 6..9: each thread copies
its next cell's state rows into shared memory with cp.async while it
integrates the current one) against the one-cell-per-thread kernels
(variant 0), for both models and both precisions, on a grid with removed
cells (compact cell indexing) and a stimulus, large enough that every block
loops over several tiles.  They run the same per-cell arithmetic, so the bar
is bit-identical V and state."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ, STEPS = 160, 160, 4, 40


def _run(model, precision, variant):
    from monoalg3d_c_b200 import Stim, Tissue
    rng = np.random.default_rng(11)
    active = (rng.random(NX * NY * NZ) >= 0.2).astype(np.uint8)
    # the CG launch shape is pinned too: the tuner's choice between shapes
    # that time alike changes V at the rounding level (their reductions add
    # in different orders)
    pinned = {"MB_ODE_VARIANT": str(variant), "MB_CG_VARIANT": "0"}
    old = {k: os.environ.get(k) for k in pinned}
    os.environ.update(pinned)
    try:
        t = Tissue(NX, NY, NZ, model=model, precision=precision, active=active,
                   stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)])
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    assert t.tuning()["ode_variant"] == variant
    t.step(STEPS)
    out = t.v(), t.state()
    t.close()
    return out


@pytest.mark.parametrize("model,precision", [("tt2006", "fp64"), ("tt2006", "mixed"),
                                             ("torord", "fp64"), ("torord", "mixed")])
def test_staged_variants_match_plain(model, precision):
    v0, s0 = _run(model, precision, 0)
    assert np.isfinite(s0).all()
    ok = np.isfinite(v0)
    for variant in (6, 7, 8, 9):
        v, s = _run(model, precision, variant)
        dv = np.abs(v[ok] - v0[ok])
        ds = np.abs(s - s0) / (np.abs(s0) + 1e-30)
        bad = np.argwhere(np.abs(s - s0) > 0)
        print(f"{model}/{precision} variant {variant}: max |dV| {dv.max():.3e} mV at {np.argmax(dv)}, "
              f"cells differing {int((dv > 0).sum())}, max rel dstate {ds.max():.3e}, "
              f"state rows differing {sorted(set(bad[:, 0].tolist()))[:10]}")
        assert np.array_equal(np.isfinite(v), ok)
        assert np.array_equal(v[ok], v0[ok]), f"{model}/{precision} variant {variant}: V differs"
        assert np.array_equal(s, s0), f"{model}/{precision} variant {variant}: state differs"

"""The resident CG kernel (cg_resident.cu: tile columns held in shared memory
and registers for the whole solve, boundary z and x exchanged through global
memory) against the flat persistent kernel and the CPU oracle, on grids that
give one and several tile columns and rows, edge tiles narrower than the
rest, removed cells, and one plane.

The kernel runs the mixed-precision solve only, so the bars are the mixed
form's: CG iteration counts within one of the flat mixed kernel's per step
(both stop on the same FP64 residual), V within 1e-4 mV of the flat mixed
kernel, and V within 0.5 mV RMS and 2e-3 relative (max) of the FP64 oracle."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

FLAT = 0                        # MB_CG_VARIANT of flat shape 0


def _resident():
    """MB_CG_VARIANT of the resident kernel (after the flat shapes and the tiled kernel)."""
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    return cg_launch_shapes() + 1


def _stims():
    from monoalg3d_c_b200 import Stim
    return [Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)]


def _run(nx, ny, nz, steps, variant, **kw):
    from monoalg3d_c_b200 import Tissue
    old = os.environ.get("MB_CG_VARIANT")
    os.environ["MB_CG_VARIANT"] = str(variant)
    try:
        t = Tissue(nx, ny, nz, precision="mixed", stims=_stims(), **kw)
    finally:
        if old is None:
            os.environ.pop("MB_CG_VARIANT", None)
        else:
            os.environ["MB_CG_VARIANT"] = old
    kernel = t.tuning()["cg_kernel"]
    t.step(steps)
    v = t.v()
    stats = t.step_stats(0, steps)
    t.close()
    return kernel, v, stats


CASES = {
    # (nx, ny, nz, steps, kwargs)
    "slab_masked": (70, 50, 6, 150, "torord_mask"),
    "odd_edges": (37, 29, 3, 150, "tt2006"),
    "sheet": (64, 48, 1, 150, "tt2006"),
    "wide_tiles": (96, 40, 4, 120, "tt2006_mask"),
}


def _kw(name, n, seed=5):
    rng = np.random.default_rng(seed)
    if name == "torord_mask":
        return dict(model="torord", assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00005,
                    active=(rng.random(n) >= 0.2).astype(np.uint8))
    if name == "tt2006_mask":
        return dict(active=(rng.random(n) >= 0.15).astype(np.uint8))
    return {}


@pytest.mark.parametrize("case", sorted(CASES))
def test_resident_matches_flat_and_oracle(case):
    nx, ny, nz, steps, kind = CASES[case]
    kw = _kw(kind, nx * ny * nz)
    k_res, v_res, s_res = _run(nx, ny, nz, steps, _resident(), **kw)
    assert k_res == 200, f"resident kernel not used ({k_res})"
    k_flat, v_flat, s_flat = _run(nx, ny, nz, steps, FLAT, **kw)
    assert k_flat == 0
    assert np.abs(s_res["its"] - s_flat["its"]).max() <= 1, "CG iteration counts differ by more than one"
    assert s_res["its"].sum() > 0
    ok = np.isfinite(v_flat)
    assert np.array_equal(ok, np.isfinite(v_res))
    d = np.abs(v_res[ok] - v_flat[ok])
    assert d.max() <= 1e-4, f"{case}: resident vs flat mixed max |dV| {d.max():.3e} mV"

    o = oracle.Sim(nx, ny, nz, stims=_stims(), **kw)
    o.step(steps)
    ref = o.v()
    o.close()
    e = v_res[ok] - ref[ok]
    rms = np.sqrt(np.mean(e ** 2))
    rel = np.max(np.abs(e) / (np.abs(ref[ok]) + 1.0))
    print(f"{case}: vs flat {d.max():.2e} mV, vs oracle RMS {rms:.2e} mV, max rel {rel:.2e}")
    assert rms <= 0.5 and rel <= 2e-3, f"{case}: vs oracle RMS {rms:.3e} mV, max rel {rel:.3e}"

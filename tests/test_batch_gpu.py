"""Batched tissues on the GPU against each tissue solved alone by the CPU
oracle (FP64): V within 1e-7 relative -- the stacked CG stops on the summed
r.r, so a tissue's solve may stop at a different iterate than its
stand-alone solve, within the 1e-16 tolerance -- and every tissue activated.
Then the mixed-precision batch against the FP64 batch (0.5 mV RMS, 0.5 ms
activation time)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def _sizes_scales(seed=12):
    rng = np.random.default_rng(seed)
    sizes = [(int(rng.integers(20, 60)), 1) for _ in range(6)] + \
            [(int(s), int(s)) for s in rng.integers(8, 24, 6)]
    scales = np.exp(0.2 * rng.standard_normal((len(sizes), 5)))
    return sizes, scales


def test_batch_matches_standalone_oracle():
    from monoalg3d_c_b200 import Stim
    from monoalg3d_c_b200.batch import Batch
    sizes, scales = _sizes_scales()
    stim = Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=300.0)
    b = Batch(sizes, scales, stim=stim, precision="fp64", track_activation=True)
    steps = 600
    b.step(steps)
    vb = b.v()
    act = b.activation()
    b.close()
    for q, (nx, ny) in enumerate(sizes):
        sc = np.repeat(np.asarray(scales[q])[:, None], nx * ny, axis=1)
        o = oracle.Sim(nx, ny, 1, current_scale=sc, stims=[stim])
        o.step(steps)
        ref = o.v().reshape(ny, nx)
        o.close()
        np.testing.assert_allclose(vb[q], ref, rtol=1e-7, atol=1e-7, err_msg=f"tissue {q} {nx}x{ny}")
        assert (act[q]["first"] >= 0).mean() > 0.9


def test_batch_mixed_against_fp64():
    from monoalg3d_c_b200 import Stim
    from monoalg3d_c_b200.batch import Batch
    sizes, scales = _sizes_scales(13)
    stim = Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=300.0)
    res = {}
    for prec in ("fp64", "mixed"):
        b = Batch(sizes, scales, stim=stim, precision=prec, track_activation=True)
        b.step(2000)
        res[prec] = (np.concatenate([v.reshape(-1) for v in b.v()]),
                     np.concatenate([a["first"].reshape(-1) for a in b.activation()]))
        b.close()
    dv = res["mixed"][0] - res["fp64"][0]
    assert np.sqrt(np.mean(dv ** 2)) <= 0.5
    on = res["fp64"][1] >= 0
    assert np.array_equal(on, res["mixed"][1] >= 0)
    assert np.abs(res["mixed"][1][on] - res["fp64"][1][on]).max() <= 0.5

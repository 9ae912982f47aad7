"""Checkpoint / restore of the loop state and V files in the reference's
save_as_text_or_binary format."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tissue(**kw):
    from monoalg3d_c_b200 import Stim, Tissue
    rng = np.random.default_rng(2)
    active = (rng.random(24 * 16 * 3) >= 0.1).astype(np.uint8)
    return Tissue(24, 16, 3, active=active, model="torord", track_activation=True,
                  stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)], **kw)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_restore_replays_the_same_steps(prec):
    t = _tissue(precision=prec)
    t.step(100)
    state = t.checkpoint()
    t.step(200)
    va, aa = t.v(), t.activation()
    t.restore(state)
    assert t.info()["count"] == 100
    t.step(200)
    vb, ab = t.v(), t.activation()
    np.testing.assert_array_equal(va, vb)
    np.testing.assert_array_equal(aa["first"], ab["first"])
    # a checkpoint belongs to its tissue's kind
    other = _tissue(precision="mixed" if prec == "fp64" else "fp64")
    from monoalg3d_c_b200 import MonoAlgError
    with pytest.raises(MonoAlgError):
        other.restore(state)
    other.close()
    t.close()


def test_save_v_text_and_binary(tmp_path):
    t = _tissue(precision="fp64")
    t.step(150)
    v = t.v()
    t.save_v(str(tmp_path / "v.txt"))
    t.save_v(str(tmp_path / "v.bin"), binary=True)
    rows = np.loadtxt(str(tmp_path / "v.txt"), delimiter=",")
    raw = np.fromfile(str(tmp_path / "v.bin"), dtype=np.float64).reshape(-1, 7)
    live = np.isfinite(v)
    assert rows.shape == (live.sum(), 7) and raw.shape == rows.shape
    np.testing.assert_array_equal(raw[:, 6], v[live])
    np.testing.assert_allclose(rows[:, 6], v[live], rtol=1e-5, atol=1e-5)
    g = np.flatnonzero(live)
    np.testing.assert_allclose(raw[:, 0], (g % 24 + 0.5) * 100.0)
    np.testing.assert_allclose(raw[:, 2], (g // (24 * 16) + 0.5) * 100.0)
    assert np.all(raw[:, 3:6] == 50.0)
    t.close()

"""Checkpoints in the reference's save_simulation_state layout
(mb_monodomain_save_state / mb_monodomain_restore_state):

  - round trip here: a tissue saved after some steps and restored into a new
    tissue holds the same V and continues as the original does, in both
    state-vector layouts (cell after cell, as the reference's CPU build
    writes it; state row after state row with the row pitch, as its GPU
    build does) and in both precisions -- to rounding, since the two
    tissues' tuners may pick different CG launch shapes (another summation
    order);
  - the reference's checkpoint, restored here: the reference runs part of
    the simulation and saves; this library restores its files and runs on,
    and matches the reference's uninterrupted run to the end (FP64 bar: 1e-8
    relative + 1e-9 mV; CG iteration counts equal step for step);
  - this library's checkpoint, restored by the reference: the reference's
    restore_simulation_state reads the files written here (cell-after-cell
    layout, as its CPU build reads them) and its run on matches this
    library's uninterrupted run.

On the benchmark workloads at reduced size: the TT2006 cuboid, the ToRORd
slab with 20 % of its cells removed (removed cells are leaves of the
reference's octree that must be matched by centre) and the z-thirds ToRORd
slab with fibres rotating through the thickness.  The interop cases need the
reference's build (oracle/_ref) on the host."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
import run_reference as rr  # noqa: E402

pytestmark = pytest.mark.gpu

REL = 1e-8
ABS = 1e-9
# benchmark configuration -> scale of the reduced tissue
CASES = {0: 0.2, 1: 0.1, 4: 0.06}


def _wl(cfg):
    from monoalg3d_c_b200 import workloads
    return workloads.CONFIGS[cfg](CASES[cfg])


def _same(a, b):
    assert np.array_equal(np.isfinite(a), np.isfinite(b))
    ok = np.isfinite(a)
    return np.array_equal(a[ok], b[ok])


@pytest.mark.parametrize("layout", ["cpu", "gpu"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("cfg", [0, 1])
def test_round_trip(tmp_path, cfg, precision, layout):
    wl = _wl(cfg)
    a = wl.tissue(precision=precision)
    a.step(60)
    a.save_state(str(tmp_path), gpu_layout=(layout == "gpu"))
    b = wl.tissue(precision=precision)
    b.restore_state(str(tmp_path))
    assert _same(a.v(), b.v())
    a.step(40)
    b.step(40)
    va, vb = a.v(), b.v()
    a.close()
    b.close()
    assert np.array_equal(np.isfinite(va), np.isfinite(vb))
    ok = np.isfinite(va)
    # FP64: rounding; mixed: the FP32 recurrences of another launch shape
    tol = 1e-12 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(vb[ok], va[ok], rtol=tol, atol=tol)


def test_restore_refuses_another_tissue(tmp_path):
    from monoalg3d_c_b200 import workloads
    a = _wl(0).tissue()
    a.step(2)
    a.save_state(str(tmp_path))
    a.close()
    other = workloads.CONFIGS[0](0.3).tissue()
    with pytest.raises(Exception):
        other.restore_state(str(tmp_path))
    other.close()


def _needs_reference():
    if not rr.available():
        pytest.skip("the reference build (oracle/_ref) is not on this host")


def _check_v(cfg, v, ref):
    ok = np.isfinite(ref)
    assert np.array_equal(ok, np.isfinite(v)), f"config {cfg}: removed cells differ"
    err = np.abs(v[ok] - ref[ok])
    assert np.all(err <= REL * np.abs(ref[ok]) + ABS), f"config {cfg}: max |dV| {err.max():.3e} mV"


# the reference runs 60 loop-step clocks, saves, and the run goes on to 110
T1, T2 = rr.sim_ms_for_steps(60), rr.sim_ms_for_steps(110)


@pytest.mark.parametrize("cfg", [0, 1, 4])
def test_reference_checkpoint_restored_here(tmp_path, cfg):
    _needs_reference()
    wl = _wl(cfg)
    case = rr.case_from_workload(wl)
    dt = case.get("dt", 0.02)
    first, total = rr.loop_steps(T1, dt), rr.loop_steps(T2, dt)
    ck = str(tmp_path / "ck")
    rr.run_case(dict(case, sim_ms=T1, save_state=dict(output_dir=ck)))
    straight = rr.run_case(dict(case, sim_ms=T2), dumps_every=10)
    last = int(straight["counts"][-1])          # V after `last` steps
    assert first < last <= total
    t = wl.tissue(precision="fp64")
    t.restore_state(ck)
    assert t.info()["count"] == first
    t.step(last - first)
    v = t.v()
    t.step(total - last)
    its = t.step_stats(first, total - first)["its"]
    t.close()
    _check_v(cfg, v, straight["V"][-1])
    np.testing.assert_array_equal(its, straight["its"][first:total])


@pytest.mark.parametrize("cfg", [0, 1, 4])
def test_checkpoint_restored_by_the_reference(tmp_path, cfg):
    _needs_reference()
    wl = _wl(cfg)
    case = rr.case_from_workload(wl)
    dt = case.get("dt", 0.02)
    first, total = rr.loop_steps(T1, dt), rr.loop_steps(T2, dt)
    a = wl.tissue(precision="fp64")
    a.step(first)
    ck = str(tmp_path / "ck")
    os.makedirs(ck)
    a.save_state(ck)
    r = rr.run_case(dict(case, sim_ms=T2, restore_state=dict(input_dir=ck)), dumps_every=10)
    last = int(r["counts"][-1])
    assert first < last <= total and len(r["its"]) == total - first
    a.step(last - first)
    v = a.v()
    a.step(total - last)
    its = a.step_stats(first, total - first)["its"]
    a.close()
    _check_v(cfg, v, r["V"][-1])
    np.testing.assert_array_equal(its, r["its"])

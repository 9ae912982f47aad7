"""Parity at the benchmark configurations' own sizes, with the launch shapes the
tissue's tuner picks there (nothing forced):

  cuboid 100x100x20, TT2006 (200 k cells), 252 steps;
  slab 200x200x50, ToRORd, fibres along x, 20 % removed (1.6 M cells), 21 steps;
  slab 500x500x100, ToRORd in z-thirds, fibres rotating through the
  thickness (25 M cells), 12 steps;

each against the reference's own CPU path (oracle/_ref, OpenMP, FP64; the
adapter plugins express the mask, the rotating fibres and the z-layers) on
the same tissue: the FP64 GPU path within 1e-8 relative (+1e-9 mV) in V at
every dump and with the reference's CG iteration count at every step, the
mixed-precision form within the 0.5 mV RMS bar; and the batching
configuration on a fixed subset of 16 of its 256 tissues (8 cables, 8
sheets, full sizes, per-tissue conductance scalings) against each tissue
solved alone by the CPU oracle (1e-7 relative: the stacked CG stops on the
summed residual).  The reference runs need its build (oracle/_ref) on the
host; they take a few minutes and, for the 25 M-cell slab, ~45 GB of host
memory."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import run_reference as rr  # noqa: E402

pytestmark = pytest.mark.gpu

REL = 1e-8
ABS = 1e-9
# configuration -> (scale, loop steps of the run, dump every)
RUNS = {0: (1.0, 252, 50), 1: (1.0, 22, 10), 4: (1.0, 12, 10)}
_cache = {}


def _needs_reference():
    if not rr.available():
        pytest.skip("the reference build (oracle/_ref) is not on this host")


def _reference(cfg: int):
    """The reference run of a configuration (computed once per session)."""
    if cfg not in _cache:
        from monoalg3d_c_b200 import workloads
        scale, steps, every = RUNS[cfg]
        wl = workloads.CONFIGS[cfg](scale)
        case = rr.case_from_workload(wl)
        case["sim_ms"] = rr.sim_ms_for_steps(steps)
        r = rr.run_case(case, dumps_every=every, timeout=3000)
        # the loop's own count for that simulation time (float clock)
        assert len(r["its"]) == rr.loop_steps(case["sim_ms"], case["dt"])
        _cache[cfg] = (wl, r)
    return _cache[cfg]


def _gpu_dumps(wl, precision, counts):
    t = wl.tissue(precision=precision)
    out, done = {}, 0
    for c in counts:
        t.step(int(c) - done)
        done = int(c)
        out[int(c)] = t.v()
    stats = t.step_stats(0, done)
    kernel = t.tuning()
    t.close()
    return out, stats, kernel


@pytest.mark.parametrize("cfg", [0, 1, 4])
def test_fp64_matches_reference_at_size(cfg):
    _needs_reference()
    wl, r = _reference(cfg)
    out, stats, kernel = _gpu_dumps(wl, "fp64", r["counts"])
    for q, c in enumerate(r["counts"]):
        ref = r["V"][q]
        ok = np.isfinite(ref)
        got = out[int(c)]
        assert np.array_equal(ok, np.isfinite(got)), f"config {cfg}: removed cells differ"
        err = np.abs(got[ok] - ref[ok])
        lim = REL * np.abs(ref[ok]) + ABS
        assert np.all(err <= lim), (f"config {cfg} step {c} ({kernel}): max |dV| {err.max():.3e} mV "
                                    f"over {ok.sum()} cells")
    n = len(stats)
    assert np.array_equal(stats["its"], r["its"][:n]), (
        f"config {cfg} ({kernel}): CG iterations {stats['its']} vs reference {r['its'][:n]}")


@pytest.mark.parametrize("cfg", [1, 4])
def test_mixed_within_bar_at_size(cfg):
    _needs_reference()
    wl, r = _reference(cfg)
    out, _, kernel = _gpu_dumps(wl, "mixed", r["counts"])
    c = int(r["counts"][-1])
    ref = r["V"][-1]
    ok = np.isfinite(ref)
    dv = out[c][ok] - ref[ok]
    rms = float(np.sqrt(np.mean(dv ** 2)))
    print(f"config {cfg} mixed ({kernel}) after {c} steps: V RMS {rms:.3e} mV, max {np.abs(dv).max():.3e} mV")
    assert rms <= 0.5


def test_batch_subset_of_the_batching_configuration():
    """16 of the batching configuration's 256 tissues (a fixed seeded choice of
    8 cables and 8 sheets at their own sizes and scalings) in one atlas,
    against each solved alone by the CPU oracle."""
    import oracle
    from monoalg3d_c_b200 import Stim, workloads
    from monoalg3d_c_b200.batch import Batch
    sizes, scales = workloads.config2_instances()
    pick = np.random.Generator(np.random.Philox(2003))
    idx = sorted(pick.choice(128, 8, replace=False).tolist()) + sorted((128 + pick.choice(128, 8, replace=False)).tolist())
    sub = [sizes[i] for i in idx]
    sc = scales[idx]
    stim = Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=100.0)
    steps = 100
    b = Batch(sub, sc, stim=stim, precision="fp64")
    b.step(steps)
    vb = b.v()
    b.close()
    for q, (nx, ny) in enumerate(sub):
        cs = np.repeat(np.asarray(sc[q])[:, None], nx * ny, axis=1)
        o = oracle.Sim(nx, ny, 1, current_scale=cs, stims=[stim])
        o.step(steps)
        ref = o.v().reshape(ny, nx)
        o.close()
        np.testing.assert_allclose(vb[q], ref, rtol=1e-7, atol=1e-7, err_msg=f"tissue {idx[q]} {nx}x{ny}")

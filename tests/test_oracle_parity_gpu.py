"""FP64 CUDA path against the CPU oracle (oracle/, pinned to the reference by
tests/test_oracle.py) on inputs the stock reference plugins cannot express:
removed (fibrotic) cells in 3-D, per-cell conductivity, fibres rotating
through the wall, z-layered ToRORd cell types, per-cell conductance
scalings, periodic and box stimuli, 1-D cables and 2-D sheets.

Bar: V within 1e-8 relative (+1e-9 mV) after every block of steps, and the
same CG iteration count per step (a step may differ by one where r.r lands
within rounding of the tolerance)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

REL = 1e-8
ABS = 1e-9


def _stim(**kw):
    from monoalg3d_c_b200 import Stim
    return Stim(**kw)


def _compare(nx, ny, nz, steps, every=50, **kw):
    from monoalg3d_c_b200 import Tissue
    kw.setdefault("stims", [_stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)])
    t = Tissue(nx, ny, nz, precision="fp64", **kw)
    o = oracle.Sim(nx, ny, nz, **kw)
    its_o = []
    done = 0
    while done < steps:
        blk = min(every, steps - done)
        for _ in range(blk):
            assert o.step(1) == 0
            its_o.append(o.last_cg()[0])
        t.step(blk)
        done += blk
        ref, got = o.v(), t.v()
        ok = np.isfinite(ref)
        assert np.array_equal(ok, np.isfinite(got)), "removed cells differ"
        err = np.abs(got[ok] - ref[ok])
        lim = REL * np.abs(ref[ok]) + ABS
        assert np.all(err <= lim), f"step {done}: max |dV| {err.max():.3e} mV"
    stats = t.step_stats(0, steps)
    t.sync()
    t.close()
    d_its = np.abs(stats["its"] - np.array(its_o))
    assert (d_its <= 1).all() and (d_its > 0).mean() < 0.05, f"CG iteration counts differ: {d_its.sum()}"
    return ref


def _fibrosis(n, frac, seed):
    return (np.random.default_rng(seed).random(n) >= frac).astype(np.uint8)


def test_tt2006_with_removed_cells():
    nx, ny, nz = 24, 16, 3
    v = _compare(nx, ny, nz, 400, active=_fibrosis(nx * ny * nz, 0.2, 5))
    assert np.nanmax(v) > 0.0           # the wave got through


def test_torord_aniso_x_with_removed_cells():
    # the precision configuration's operator: fibres along x, 20 % removed
    nx, ny, nz = 20, 12, 3
    _compare(nx, ny, nz, 250, model="torord", assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00005,
             active=_fibrosis(nx * ny * nz, 0.2, 6))


def test_per_cell_sigma_with_removed_cells():
    nx, ny, nz = 20, 20, 1
    rng = np.random.default_rng(7)
    sig = 0.00013 * np.exp(0.3 * rng.standard_normal(nx * ny * nz))
    _compare(nx, ny, nz, 300, assembly="per_cell", sigma_cell=sig, active=_fibrosis(nx * ny * nz, 0.1, 8))


def test_rotating_fibres_transmural_torord():
    # the scale configuration's operator and cell layering on a small slab
    nx, ny, nz = 16, 12, 6
    ang = np.deg2rad(np.linspace(60.0, -60.0, nz))
    ct = np.repeat(np.array([0, 0, 1, 1, 2, 2], dtype=np.uint8), nx * ny)
    stims = [_stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0),
             _stim(kind="x_y_limits", start=3.0, duration=2.0, current=-53.0, min=(0.0, 0.0, 0.0),
                   max=(800.0, 600.0, 0.0))]
    _compare(nx, ny, nz, 300, model="torord", assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00004,
             fibre_angle_z=ang, celltype=ct, stims=stims)


def test_tt2006_conductance_scalings():
    nx, ny, nz = 30, 10, 1
    rng = np.random.default_rng(9)
    scale = np.exp(0.2 * rng.standard_normal((5, nx * ny * nz)))
    _compare(nx, ny, nz, 300, current_scale=scale)


def test_torord_scalings_and_true_rl_rule():
    nx, ny, nz = 12, 8, 2
    rng = np.random.default_rng(10)
    scale = np.exp(0.2 * rng.standard_normal((5, nx * ny * nz)))
    _compare(nx, ny, nz, 200, model="torord", rl_rule="true", current_scale=scale)


def test_cable_periodic_stimulus():
    # 1-D cable stimulated at its x = 0 end every 4 ms (the later pulses fall
    # in the refractory period; they exercise the period shift)
    stims = [_stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0, period=4.0)]
    v = _compare(100, 1, 1, 700, stims=stims)
    assert np.nanmax(v) > 0.0


def test_ode_substeps():
    # dt_ode = dt_pde / 4: four Rush-Larsen sub-steps per loop step
    _compare(16, 8, 1, 150, dt_pde=0.04, dt_ode=0.01)

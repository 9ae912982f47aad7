"""The CPU oracle (oracle/, a C restatement of the reference path) pinned
against the reference's own CPU build: the golden fixtures under
tests/golden/ were made by running the reference MonoAlg3D (make_golden.py).

Bar: the same as for the CUDA path -- V within 1e-8 relative at every dump
and the same CG iteration count per step (a step may differ by one where the
reference's r.r lands within rounding of the tolerance).  Plus unit checks of
the restated pieces: the matrix (symmetric, row sums = alpha on interior
cells, removed cells decoupled) and the CG against a dense solve."""
import os
import sys

import numpy as np
import pytest

import golden_cases as gc

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

REL = 1e-8
ABS = 1e-9


@pytest.mark.parametrize("name", gc.CASE_NAMES)
def test_oracle_matches_reference(name):
    g = gc.load(name)
    cfg = g["config"]
    sim = oracle.Sim(cfg["nx"], cfg["ny"], cfg["nz"], **gc.tissue_kwargs(cfg))
    done = 0
    its = []
    counts = [int(c) for c in g["counts"]]
    q = 0
    for step in range(len(g["its"])):
        if q < len(counts) and counts[q] == step:
            ref = g["V"][q]
            got = sim.v()
            ok = np.isfinite(ref)          # removed cells read NaN in both
            assert np.array_equal(ok, np.isfinite(got)), f"{name}: removed cells differ"
            err = np.abs(got[ok] - ref[ok])
            lim = REL * np.abs(ref[ok]) + ABS
            assert np.all(err <= lim), f"{name} step {step}: max |dV| {err.max():.3e} mV"
            q += 1
        assert sim.step(1) == 0
        its.append(sim.last_cg()[0])
        done += 1
    d_its = np.abs(np.array(its) - g["its"])
    assert (d_its <= 1).all() and (d_its > 0).mean() < 0.02, f"{name}: CG iteration counts differ: {d_its.sum()}"


def test_loop_steps_match_reference_count():
    # 12 ms at dt 0.02: the reference loop runs while cur_time - T <= dt
    assert oracle.loop_steps(12.0, 0.02) == len(gc.load("tt2006_cuboid")["its"])


def _dense(rp, col, val):
    n = rp.size - 1
    A = np.zeros((n, n))
    for i in range(n):
        for e in range(rp[i], rp[i + 1]):
            A[i, col[e]] += val[e]
    return A


@pytest.mark.parametrize("aniso", [False, True])
def test_matrix_properties_with_removed_cells(aniso):
    nx, ny, nz = 7, 6, 4
    rng = np.random.default_rng(3)
    active = (rng.random(nx * ny * nz) >= 0.25).astype(np.uint8)
    kw = dict(active=active)
    if aniso:
        kw.update(assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00005,
                  fibre_angle_z=np.linspace(np.pi / 3, -np.pi / 3, nz))
    rp, col, val, cells = oracle.assemble(nx, ny, nz, **kw)
    A = _dense(rp, col, val)
    assert cells.size == active.sum()
    if not aniso:
        # the face-flux scheme is symmetric; the reference's anisotropic scheme,
        # whose cross terms average over whichever neighbours exist, is not
        np.testing.assert_allclose(A, A.T, rtol=0, atol=1e-15)
    alpha = ((0.14 * 1.0) / 0.02) * float(np.float32(1e-8)) * 1e6
    # every row of alpha I + K sums to alpha (K has zero row sums: no-flux at
    # the domain boundary and at removed cells)
    np.testing.assert_allclose(A.sum(axis=1), alpha, rtol=0, atol=1e-13)
    # the diagonal comes first in every row
    assert all(col[rp[i]] == i for i in range(cells.size))
    if not aniso:
        assert np.all(np.linalg.eigvalsh(A) > 0)


def test_pcg_against_dense_solve():
    rp, col, val, cells = oracle.assemble(9, 7, 3, assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00005,
                                          fibre_angle_z=np.full(3, 0.5))
    A = _dense(rp, col, val)
    rng = np.random.default_rng(11)
    b = rng.standard_normal(cells.size)
    x, its, err = oracle.pcg(rp, col, val, b, np.zeros_like(b), tol=1e-24, max_its=500)
    np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=1e-10, atol=1e-12)
    assert err <= 1e-24 and 1 < its < 500


def test_ecg_restatement_matches_reference():
    """The oracle's pseudo-bidomain ECG, evaluated on the reference's own V
    dumps, against the ecg.txt the reference wrote at the same steps (its
    "%lf" output: six decimals)."""
    import json
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tt2006_ecg.npz"))
    cfg = json.loads(str(g["config"]))
    e = cfg["ecg"]
    rate = e["calc_rate"]
    checked = 0
    for c, v in zip(g["counts"], g["V"]):
        if c % rate:
            continue
        got = oracle.pseudo_bidomain_ecg(v, cfg["nx"], cfg["ny"], cfg["nz"], e["leads"], e["sigma_b"])
        ref = g["ecg"][c // rate]
        assert np.allclose(got, ref, rtol=0, atol=6e-7), f"count {c}: {got} vs {ref}"
        checked += 1
    assert checked >= 20
    assert np.abs(g["ecg"]).max() > 0.5        # the wave's signal, not only zeros


def _tangent_problem():
    from monoalg3d_c_b200 import Stim
    nx, ny, steps, every = 10, 8, 300, 50
    rng = np.random.default_rng(3)
    n = nx * ny
    sigma = 0.00013 * np.exp(0.3 * rng.standard_normal(n))
    gkr = np.exp(0.2 * rng.standard_normal(n))
    sensors = rng.choice(n, size=6, replace=False)
    kw = dict(stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)],
              cg_tolerance=1e-24, cg_max_iterations=500, assembly="per_cell")
    return nx, ny, steps, every, sigma, gkr, sensors, kw, rng


def _scales(gkr):
    sc = np.ones((5, gkr.size))
    sc[1] = gkr
    return sc


def _oracle_misfit(nx, ny, steps, every, sigma, gkr, sensors, kw, target):
    o = oracle.Sim(nx, ny, 1, sigma_cell=sigma, current_scale=_scales(gkr), **kw)
    tr = []
    for _ in range(steps // every):
        o.step(every)
        tr.append(o.v()[sensors])
    o.close()
    tr = np.array(tr)
    return tr, 0.5 * float(np.sum((tr - target) ** 2))


def test_tangent_linear_loop_matches_oracle_differences():
    """The tangent-linear loop (tangent.cc) against central differences of the
    oracle loop: its misfit equals the loop's, and its directional derivatives
    along a conductivity and a gKr direction agree to 1e-6 relative (the
    differences' own truncation error: h^2 ~ 1e-8 for the conductivity; the gKr
    scaling is applied as a float, so its differences use the rounded values)."""
    nx, ny, steps, every, sigma, gkr, sensors, kw, rng = _tangent_problem()
    target, _ = _oracle_misfit(nx, ny, steps, every, sigma * 0.8, gkr, sensors, kw, 0.0)
    _, loss = _oracle_misfit(nx, ny, steps, every, sigma, gkr, sensors, kw, target)
    d = rng.standard_normal(sigma.size)
    tl_loss, tl_d = oracle.tangent_misfit(nx, ny, 1, steps, every, sensors, target, dsigma=sigma * d,
                                          sigma_cell=sigma, current_scale=_scales(gkr), **kw)
    assert abs(tl_loss - loss) <= 1e-12 * abs(loss)
    h = 1e-4
    fd = (_oracle_misfit(nx, ny, steps, every, sigma * (1 + h * d), gkr, sensors, kw, target)[1] -
          _oracle_misfit(nx, ny, steps, every, sigma * (1 - h * d), gkr, sensors, kw, target)[1]) / (2 * h)
    assert abs(tl_d - fd) <= 1e-6 * abs(fd), f"sigma: tangent {tl_d:.12e}, differences {fd:.12e}"
    dg = rng.standard_normal(gkr.size)
    kp = np.float32(gkr * (1 + 1e-3 * dg)).astype(np.float64)
    km = np.float32(gkr * (1 - 1e-3 * dg)).astype(np.float64)
    fd = (_oracle_misfit(nx, ny, steps, every, sigma, kp, sensors, kw, target)[1] -
          _oracle_misfit(nx, ny, steps, every, sigma, km, sensors, kw, target)[1]) / 2.0
    _, tl_g = oracle.tangent_misfit(nx, ny, 1, steps, every, sensors, target, dgkr=(kp - km) / 2.0,
                                    sigma_cell=sigma, current_scale=_scales(gkr), **kw)
    assert abs(tl_g - fd) <= 1e-6 * abs(fd), f"gKr: tangent {tl_g:.12e}, differences {fd:.12e}"

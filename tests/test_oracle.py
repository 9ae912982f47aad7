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
            err = np.abs(got - ref)
            lim = REL * np.abs(ref) + ABS
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

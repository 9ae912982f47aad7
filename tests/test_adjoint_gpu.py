"""Discrete adjoint of the loop (mb_adjoint_*): gradients of an L2 misfit of V
at sensor cells with respect to the per-cell conductivity and gKr scaling,
against central finite differences of the same FP64 GPU loop along random
directions, against central differences of the CPU oracle (FP64), against
the oracle's FP64 tangent-linear loop (exact directional derivatives), and
through the torch.autograd.Function.

Bar: directional derivatives within 1e-4 relative of the finite differences,
within 1e-6 relative of the tangent-linear derivatives.
The loop's CG tolerance is tightened to 1e-24 so that the solves' own error
does not dominate the differences; the gKr scaling is applied as a float, so
its differences use the float-rounded perturbed values."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

REL = 1e-4


def _problem(nx=16, ny=16, steps=400, seed=0):
    rng = np.random.default_rng(seed)
    n = nx * ny
    sigma = 0.00013 * np.exp(0.3 * rng.standard_normal(n))
    gkr = np.exp(0.2 * rng.standard_normal(n))
    sensors = rng.choice(n, size=6, replace=False)
    return nx, ny, steps, sigma, gkr, sensors


def _kw():
    from monoalg3d_c_b200 import Stim
    return dict(stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)],
                cg_tolerance=1e-24, cg_max_iterations=500)


def _rounded(x):
    return np.float32(x).astype(np.float64)


def test_gradients_match_gpu_finite_differences():
    from monoalg3d_c_b200.adjoint import Adjoint
    nx, ny, steps, sigma, gkr, sensors = _problem()
    adj = Adjoint(nx, ny, 1, sigma, gkr, sensors, nsteps=steps, sample_every=50, checkpoint_every=50, **_kw())
    target = adj.forward(sigma * 1.2, gkr * 0.9)
    tr = adj.forward(sigma, gkr)
    loss = lambda t: 0.5 * np.sum((t - target) ** 2)  # noqa: E731
    gs, gk = adj.backward(tr - target)
    rng = np.random.default_rng(5)
    for trial in range(3):
        d = rng.standard_normal(sigma.size)
        h = 1e-4
        lp = loss(adj.forward(sigma * (1 + h * d), gkr))
        lm = loss(adj.forward(sigma * (1 - h * d), gkr))
        fd = (lp - lm) / (2 * h)
        ad = np.sum(gs * sigma * d)
        assert abs(ad - fd) <= REL * abs(fd), f"sigma direction {trial}: adjoint {ad:.10e}, fd {fd:.10e}"
    for trial in range(3):
        d = rng.standard_normal(gkr.size)
        h = 1e-2
        kp, km = _rounded(gkr * (1 + h * d)), _rounded(gkr * (1 - h * d))
        lp = loss(adj.forward(sigma, kp))
        lm = loss(adj.forward(sigma, km))
        fd = (lp - lm) / 2.0
        ad = np.sum(gk * (kp - km)) / 2.0
        assert abs(ad - fd) <= REL * abs(fd) + 1e-12, f"gKr direction {trial}: adjoint {ad:.10e}, fd {fd:.10e}"
    adj.close()


def _oracle_traces(nx, ny, steps, sigma, gkr, sensors, every):
    sc = np.ones((5, nx * ny))
    sc[1] = gkr
    o = oracle.Sim(nx, ny, 1, assembly="per_cell", sigma_cell=sigma, current_scale=sc, **_kw())
    out = []
    for s in range(steps // every):
        o.step(every)
        out.append(o.v()[sensors])
    o.close()
    return np.array(out)


def test_gradients_match_cpu_oracle_differences():
    from monoalg3d_c_b200.adjoint import Adjoint
    nx, ny, steps, sigma, gkr, sensors = _problem(10, 8, 300, seed=3)
    adj = Adjoint(nx, ny, 1, sigma, gkr, sensors, nsteps=steps, sample_every=50, checkpoint_every=40, **_kw())
    target = _oracle_traces(nx, ny, steps, sigma * 0.8, gkr, sensors, 50)
    tr = adj.forward(sigma, gkr)
    np.testing.assert_allclose(tr, _oracle_traces(nx, ny, steps, sigma, gkr, sensors, 50), rtol=1e-8, atol=1e-9)
    gs, gk = adj.backward(tr - target)
    adj.close()
    loss = lambda t: 0.5 * np.sum((t - target) ** 2)  # noqa: E731
    rng = np.random.default_rng(8)
    d = rng.standard_normal(sigma.size)
    h = 1e-4
    fd = (loss(_oracle_traces(nx, ny, steps, sigma * (1 + h * d), gkr, sensors, 50)) -
          loss(_oracle_traces(nx, ny, steps, sigma * (1 - h * d), gkr, sensors, 50))) / (2 * h)
    ad = np.sum(gs * sigma * d)
    assert abs(ad - fd) <= REL * abs(fd), f"sigma: adjoint {ad:.10e}, oracle fd {fd:.10e}"
    d = rng.standard_normal(gkr.size)
    kp, km = _rounded(gkr * (1 + 1e-2 * d)), _rounded(gkr * (1 - 1e-2 * d))
    fd = (loss(_oracle_traces(nx, ny, steps, sigma, kp, sensors, 50)) -
          loss(_oracle_traces(nx, ny, steps, sigma, km, sensors, 50))) / 2.0
    ad = np.sum(gk * (kp - km)) / 2.0
    assert abs(ad - fd) <= REL * abs(fd) + 1e-12, f"gKr: adjoint {ad:.10e}, oracle fd {fd:.10e}"


def test_gradients_match_cpu_tangent_linear():
    from monoalg3d_c_b200.adjoint import Adjoint
    nx, ny, steps, sigma, gkr, sensors = _problem(10, 8, 300, seed=3)
    adj = Adjoint(nx, ny, 1, sigma, gkr, sensors, nsteps=steps, sample_every=50, checkpoint_every=40, **_kw())
    target = _oracle_traces(nx, ny, steps, sigma * 0.8, gkr, sensors, 50)
    tr = adj.forward(sigma, gkr)
    gs, gk = adj.backward(tr - target)
    adj.close()
    sc = np.ones((5, nx * ny))
    sc[1] = gkr
    tl = dict(assembly="per_cell", sigma_cell=sigma, current_scale=sc, **_kw())
    rng = np.random.default_rng(11)
    for trial in range(2):
        d = rng.standard_normal(sigma.size)
        _, tl_d = oracle.tangent_misfit(nx, ny, 1, steps, 50, sensors, target, dsigma=sigma * d, **tl)
        ad = np.sum(gs * sigma * d)
        assert abs(ad - tl_d) <= 1e-6 * abs(tl_d), f"sigma {trial}: adjoint {ad:.12e}, tangent {tl_d:.12e}"
        dg = rng.standard_normal(gkr.size)
        _, tl_g = oracle.tangent_misfit(nx, ny, 1, steps, 50, sensors, target, dgkr=gkr * dg, **tl)
        ad = np.sum(gk * gkr * dg)
        assert abs(ad - tl_g) <= 1e-6 * abs(tl_g), f"gKr {trial}: adjoint {ad:.12e}, tangent {tl_g:.12e}"


def test_autograd_function():
    import torch
    from monoalg3d_c_b200.adjoint import Adjoint, traces
    nx, ny, steps, sigma, gkr, sensors = _problem(12, 12, 200, seed=4)
    adj = Adjoint(nx, ny, 1, sigma, gkr, sensors, nsteps=steps, sample_every=50, checkpoint_every=50, **_kw())
    target = torch.from_numpy(adj.forward(sigma * 1.1, gkr))
    s = torch.tensor(sigma, requires_grad=True)
    k = torch.tensor(gkr, requires_grad=True)
    loss = 0.5 * ((traces(s, k, adj) - target) ** 2).sum()
    loss.backward()
    tr = adj.forward(sigma, gkr)
    gs, gk = adj.backward(tr - target.numpy())
    np.testing.assert_allclose(s.grad.numpy(), gs, rtol=1e-12, atol=0)
    np.testing.assert_allclose(k.grad.numpy(), gk, rtol=1e-12, atol=0)
    assert np.abs(gs).max() > 0 and np.abs(gk).max() > 0
    adj.close()


def test_mixed_forward_adjoint():
    """The configuration's form: FP32 forward (mixed cell model and CG), FP64
    accumulation of the adjoint and the gradients.  Its directional
    derivatives against the FP64 adjoint's at the same point (1e-3 of the
    summed magnitudes of the direction's terms, sum |g d|: the Jacobian is
    formed in FP32, and a random direction's derivative can cancel to far
    below its terms), and central differences of the mixed loop
    at a step of 1e-2 in sigma (the FP32 forward's rounding limits how small
    the step can be; at that step the differences of this small sheet carry a
    few per cent of curvature) against those of the FP64 loop at the same
    step (1e-2), with the mixed adjoint no further from the mixed loop's
    differences than the FP64 adjoint is from the FP64 loop's, plus 1e-2."""
    from monoalg3d_c_b200.adjoint import Adjoint
    nx, ny, steps, sigma, gkr, sensors = _problem()
    a64 = Adjoint(nx, ny, 1, sigma, gkr, sensors, nsteps=steps, sample_every=50, checkpoint_every=50, **_kw())
    am = Adjoint(nx, ny, 1, sigma, gkr, sensors, nsteps=steps, sample_every=50, checkpoint_every=50,
                 precision="mixed", **_kw())
    target = a64.forward(sigma * 1.2, gkr * 0.9)
    loss = lambda t: 0.5 * np.sum((t - target) ** 2)  # noqa: E731
    t64 = a64.forward(sigma, gkr)
    g64s, g64k = a64.backward(t64 - target)
    tm = am.forward(sigma, gkr)
    gms, gmk = am.backward(tm - target)
    rng = np.random.default_rng(11)
    h = 1e-2
    for trial in range(3):
        d = rng.standard_normal(sigma.size)
        dm, d64 = float(np.sum(gms * sigma * d)), float(np.sum(g64s * sigma * d))
        fdm = (loss(am.forward(sigma * (1 + h * d), gkr)) - loss(am.forward(sigma * (1 - h * d), gkr))) / (2 * h)
        fd64 = (loss(a64.forward(sigma * (1 + h * d), gkr)) - loss(a64.forward(sigma * (1 - h * d), gkr))) / (2 * h)
        print(f"sigma direction {trial}: mixed adjoint {dm:.6e}, FP64 adjoint {d64:.6e}, "
              f"mixed FD {fdm:.6e}, FP64 FD {fd64:.6e}")
        assert abs(dm - d64) <= 1e-3 * float(np.sum(np.abs(g64s * sigma * d)))
        assert abs(fdm - fd64) <= 1e-2 * abs(fd64)
        assert abs(dm - fdm) <= abs(d64 - fd64) + 1e-2 * abs(fd64)
        dk = rng.standard_normal(sigma.size)
        km, k64 = float(np.sum(gmk * dk)), float(np.sum(g64k * dk))
        print(f"gKr direction {trial}: mixed adjoint {km:.6e}, FP64 adjoint {k64:.6e}")
        assert abs(km - k64) <= 1e-3 * float(np.sum(np.abs(g64k * dk)))
    a64.close()
    am.close()

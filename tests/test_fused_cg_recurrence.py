"""The fused mixed CG iteration of the z-march kernel (cg_zmarch.cu, FUSED
variants) at the level of vectors, on the CPU: FP32 r, p and A p, FP64 x and
dot products, FP64 true-residual refinement.  One pass per iteration forms
r_k = r_{k-1} - a A p_{k-1} and p_k = z_k + beta p_{k-1}, and sums p.q, q.z,
q.Mq, q.r, q.q and the stored r_k's own r.z and r.r; the next r.z and r.r
come from `r.z - 2 a q.z + a^2 q.Mq` with a = alpha rounded to FP32.  Checked
against the two-pass loop (Q then U, r.z and r.r summed from the stored r)
on random SPD systems with a dominant diagonal like the monodomain
operator's: the same iteration counts and refinement points, the same
tolerance met.  A variant that carries the predicted r.z from iteration to
iteration instead of restarting it from the stored r's sums is shown to
drift (the failure mode the kernel avoids)."""
import numpy as np
import pytest

F = np.float32


def _system(seed, n=300):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n)) * 0.05
    A = B @ B.T + np.diag(5.0 + rng.random(n))
    return A, rng.standard_normal(n), rng.standard_normal(n)


def _resid(A, b, x, minv):
    r64 = b - A @ x
    rt = r64.astype(F)
    z = minv * rt
    return rt, float(rt.astype(float) @ z.astype(float)), float(rt.astype(float) @ rt.astype(float)), float(r64 @ r64)


def two_pass(A, b, x, tol=1e-20, ratio=1e-10, floor=1e-22, max_its=200):
    minv = (1.0 / np.diag(A)).astype(F)
    A32 = A.astype(F)
    r, rz, rr, e = _resid(A, b, x, minv)
    rr_ref, its, first, beta, p, refine_at = e, 1, True, 0.0, np.zeros(len(b), F), []
    done = e < tol
    while not done:
        z = minv * r
        p = z if first else (F(beta) * p + z).astype(F)
        q = (A32 @ p).astype(F)
        alpha = rz / float(p.astype(float) @ q.astype(float))
        x = x + alpha * p.astype(float)
        r = (r - F(alpha) * q).astype(F)
        z = minv * r
        rzn, rrn = float(r.astype(float) @ z.astype(float)), float(r.astype(float) @ r.astype(float))
        its += 1
        if rrn <= max(floor, ratio * rr_ref) or its >= max_its:
            r, rz, rr, e = _resid(A, b, x, minv)
            rr_ref, first = e, True
            refine_at.append(its)
            done = e <= tol or its >= max_its
        else:
            beta, rz, rr, first = rzn / rz, rzn, rrn, False
    return x, its, refine_at, e


def fused(A, b, x, tol=1e-20, ratio=1e-10, floor=1e-22, max_its=200, restart_sums=True):
    minv = (1.0 / np.diag(A)).astype(F)
    A32 = A.astype(F)
    r, rz, rr, e = _resid(A, b, x, minv)
    rr_ref, its, first, xupd, alpha, beta, refine_at = e, 1, True, False, 0.0, 0.0, []
    p, q = np.zeros(len(b), F), np.zeros(len(b), F)
    done = e < tol
    while not done:
        if xupd:
            x = x + alpha * p.astype(float)          # the previous direction, a pass late
        if not first:
            r = (r - F(alpha) * q).astype(F)
        z = minv * r
        p = z if first else (F(beta) * p + z).astype(F)
        q = (A32 @ p).astype(F)
        qd, rd = q.astype(float), r.astype(float)
        s = [p.astype(float) @ qd, qd @ z.astype(float), qd @ (minv * q).astype(float), qd @ rd, qd @ qd,
             rd @ z.astype(float), rd @ rd]
        if restart_sums:
            rz, rr = s[5], s[6]
        alpha = rz / s[0]
        a = float(F(alpha))
        rz_n = rz - 2 * a * s[1] + a * a * s[2]
        rr_n = rr - 2 * a * s[3] + a * a * s[4]
        xupd, its = True, its + 1
        if rr_n <= max(floor, ratio * rr_ref) or its >= max_its:
            r, rz, rr, e = _resid(A, b, x + alpha * p.astype(float), minv)
            rr_ref, first = e, True
            refine_at.append(its)
            done = e <= tol or its >= max_its
        else:
            beta, rz, rr, first = rz_n / rz, rz_n, rr_n, False
    if xupd:
        x = x + alpha * p.astype(float)
    return x, its, refine_at, e


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_fused_matches_two_pass(seed):
    A, b, x0 = _system(seed)
    x2, its2, ref2, e2 = two_pass(A, b, x0)
    xf, itsf, reff, ef = fused(A, b, x0)
    assert ef <= 1e-20 and e2 <= 1e-20
    assert itsf == its2 and reff == ref2
    assert np.linalg.norm(b - A @ xf) ** 2 == pytest.approx(ef, rel=1e-6, abs=1e-24)
    assert np.allclose(xf, x2, rtol=1e-9, atol=1e-12)


def test_carried_recurrence_drifts():
    # carrying the predicted r.z across iterations accumulates the rounding
    # of every stored r: the solve takes longer or fails to converge
    A, b, x0 = _system(0)
    _, its_ok, _, e_ok = fused(A, b, x0)
    with np.errstate(all="ignore"):
        _, its_bad, _, e_bad = fused(A, b, x0, restart_sums=False, max_its=60)
    assert e_ok <= 1e-20
    assert its_bad > its_ok or not (e_bad <= 1e-20)

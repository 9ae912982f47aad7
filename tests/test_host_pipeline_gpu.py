"""The pipelined reference-host steps (mb_monodomain_step_host_async: stimulus
in and V out on a copy stream under the neighbouring steps' compute, two
host buffer pairs) against the synchronous call (mb_monodomain_step_host)
on the same tissue and the same per-step stimulus: the V delivered to the
host after every step is bit-identical.  The stimulus changes from step to
step, so a copy into the wrong slot or a V read too early would show."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ, STEPS = 40, 24, 4, 60


def _tissue(precision):
    import os
    from monoalg3d_c_b200 import Tissue
    rng = np.random.default_rng(9)
    active = (rng.random(NX * NY * NZ) >= 0.2).astype(np.uint8)
    # both tissues take the same launch shapes (the tuners' choices between
    # shapes that time alike differ at the rounding level)
    pinned = {"MB_ODE_VARIANT": "0", "MB_CG_VARIANT": "0"}
    old = {k: os.environ.get(k) for k in pinned}
    os.environ.update(pinned)
    try:
        t = Tissue(NX, NY, NZ, active=active, precision=precision, model="tt2006")
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return t, active


def _stim(step, n_active):
    s = np.zeros(n_active)
    if step < 100:
        s[: n_active // 5] = -53.0 * (1.0 + 0.01 * step)
    s[(7 * step) % n_active] += -20.0
    return s


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pipelined_host_steps_match_synchronous(precision):
    import torch
    from monoalg3d_c_b200 import _lib
    lib = _lib.lib
    ta, active = _tissue(precision)
    tb, _ = _tissue(precision)
    na = int(active.sum())
    n = NX * NY * NZ
    ref = []
    for k in range(STEPS):
        st = np.ascontiguousarray(_stim(k, na))
        v = np.empty(n)
        _lib.check(lib.mb_monodomain_step_host(ta._h, st.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)))
        ref.append(v)
    stim = [torch.zeros(na, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    vout = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    got = []
    for k in range(STEPS):
        s = k % 2
        # slot s was last used by call k - 2, whose copies call k - 1 waited for
        stim[s].numpy()[:] = _stim(k, na)
        _lib.check(lib.mb_monodomain_step_host_async(tb._h, C.c_void_p(stim[s].data_ptr()),
                                                     C.c_void_p(vout[s].data_ptr())))
        if k >= 1:
            # the call returned: the copies of call k - 1 (the other slot) are done
            got.append(vout[1 - s].numpy().copy())
    _lib.check(lib.mb_monodomain_host_wait(tb._h))
    got.append(vout[(STEPS - 1) % 2].numpy().copy())
    assert len(got) == STEPS
    for k in range(STEPS):
        a, b = ref[k], got[k]
        ok = np.isfinite(a)
        assert np.array_equal(ok, np.isfinite(b)), f"step {k}: removed cells differ"
        assert np.array_equal(a[ok], b[ok]), f"step {k}: max |dV| {np.abs(a[ok] - b[ok]).max():.3e}"
    ta.close()
    tb.close()

"""V in and out of the cell-model state (mb_ode_set_v / mb_ode_get_v, the
calls the reference-host plugins make every step): contiguous V (stride 1,
copied straight from and to the caller's buffer) and V inside an AoS state
array (stride neq, gathered and scattered on the host) move the same values
into the state's V row and back, and leave the other state rows alone."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


@pytest.mark.parametrize("stride", [1, 19])
def test_v_round_trip(stride):
    from monoalg3d_c_b200 import OdeSolver
    from monoalg3d_c_b200._lib import check, lib
    n = 5003
    o = OdeSolver("tt2006", n, 0.02)
    o.set_model_initial_conditions_gpu()
    before = o.state()
    rng = np.random.default_rng(7)
    v = rng.uniform(-90.0, 40.0, n)
    buf = np.zeros(n * stride)
    buf[::stride] = v
    check(lib.mb_ode_set_v(o._h, _ptr(buf), stride))
    after = o.state()
    np.testing.assert_array_equal(after[0], v)
    np.testing.assert_array_equal(after[1:], before[1:])
    out = np.full(n * stride, 123.0)
    check(lib.mb_ode_get_v(o._h, _ptr(out), stride))
    np.testing.assert_array_equal(out[::stride], v)
    if stride > 1:
        mask = np.ones(n * stride, bool)
        mask[::stride] = False
        assert np.all(out[mask] == 123.0)
    o.close()

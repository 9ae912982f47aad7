"""The forward-Euler library ToRORd_fkatp_endo, host side: the initial state
the product starts from is the library's own (read from the reference build
into tests/golden/torord_endo_steps.npz), and the fixtures of the GPU parity
tests are complete."""
import numpy as np

import golden_cases as gc


def test_initial_state_is_the_libraries():
    from monoalg3d_c_b200.monodomain import init_cell_model_data, torord_endo_initial_state
    z = np.load(f"{gc.GOLDEN}/torord_endo_steps.npz")
    assert np.array_equal(torord_endo_initial_state(), z["initial_state"])
    neq, v0 = init_cell_model_data("torord_endo")
    assert neq == 43 and v0 == z["initial_state"][0]
    gpu = torord_endo_initial_state(gpu_build=True)
    assert gpu.shape == (43,) and gpu[0] != v0       # the GPU build starts from another state


def test_fixtures():
    for name in gc.ENDO_CASE_NAMES:
        g = gc.load(name)
        assert np.isfinite(g["V"]).all()
        assert len(g["its"]) > 0 and g["counts"][0] == 0
        assert g["V"][-1].max() > 0.0       # the wave has started

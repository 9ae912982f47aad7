"""CPU checks of the C-ABI library: it loads, exports every symbol the public
header declares, and its host-side helpers follow the reference."""
import os
import re

import numpy as np

import golden_cases as gc

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(REPO, "include", "monoalg3d_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mb_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    import ctypes
    from monoalg3d_c_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    decl = _declared()
    assert len(decl) >= 25
    missing = [s for s in decl if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == decl


def test_cell_model_data():
    from monoalg3d_c_b200 import init_cell_model_data
    neq, v0 = init_cell_model_data("tt2006")
    assert neq == 19 and v0 == np.float32(-85.23)
    neq, v0 = init_cell_model_data("torord")
    assert neq == 43 and v0 == -88.7638


def test_loop_step_count_matches_reference_runs():
    from monoalg3d_c_b200 import loop_steps
    for name in gc.CASE_NAMES:
        g = gc.load(name)
        assert loop_steps(g["config"]["sim_ms"], g["config"]["dt"]) == len(g["its"])
    assert loop_steps(100.0, 0.02) == 5002
    assert loop_steps(200.0, 0.02) == 10001
    assert loop_steps(500.0, 0.02) == 25002


def test_no_device_reports_error_not_fallback():
    """Without a GPU the library reports a CUDA error instead of computing on the host."""
    from monoalg3d_c_b200 import MonoAlgError, Tissue, device_count
    if device_count() > 0:
        return
    try:
        Tissue(4, 4, 1)
    except MonoAlgError as e:
        assert e.code in (2, 4)
    else:
        raise AssertionError("tissue created without a device")

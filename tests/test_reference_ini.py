"""The reference-runner's ini text (oracle/ref/run_reference.py, test
infrastructure): the drop-in measurement names this library's reference-host
plugins in place of the stock cell model and linear solver, in the CPU and
the GPU build's library folders, and leaves every other plugin stock."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle", "ref"))
import run_reference as rr  # noqa: E402


def _case(**kw):
    return dict(nx=8, ny=4, nz=2, model="tt2006", assembly="homogeneous", sim_ms=0.1, **kw)


def test_plugin_lib_replaces_model_and_solver():
    lib = "/somewhere/libmb_shim_tt2006.so"
    for gpu in (False, True):
        libs = rr.CUDA_LIBS if gpu else rr.LIBS
        stock = rr.ini_text(_case(use_gpu=gpu), "/tmp")
        text = rr.ini_text(_case(use_gpu=gpu, plugin_lib=lib), "/tmp")
        assert f"library_file={libs}/{rr.MODEL_LIBS['tt2006']}" in stock
        assert f"library_file={libs}/libdefault_linear_system_solver.so" in stock
        assert f"library_file={libs}/{rr.MODEL_LIBS['tt2006']}" not in text
        assert f"library_file={libs}/libdefault_linear_system_solver.so" not in text
        assert text.count(f"library_file={lib}") == 2
        # everything else is the stock ini
        assert text.replace(f"library_file={lib}", "") == stock.replace(
            f"library_file={libs}/{rr.MODEL_LIBS['tt2006']}", "").replace(
            f"library_file={libs}/libdefault_linear_system_solver.so", "")

"""Drop-in test: the unmodified reference MonoAlg3D binary (its CPU build,
oracle/_ref, built from its own sources) runs its own time loop twice on the
same ini, once with its stock cell-model and linear-solver plugins and once
with this library's reference-host plugins (monoalg3d_c_b200/shim: the
same entry points, the ODE and CG work on the GPU) named in [ode_solver]
and [linear_system_solver] library_file.  The V dumps (the binary layout of
the reference's save_as_text_or_binary, every 10 steps) and the CG iteration
counts of every step of the two runs are compared.  Bar: V within 1e-8 relative (FP64), identical iteration
counts.

The same comparison runs the reference's GPU build (oracle/_ref/cuda, built
by Makefile.cuda) with [ode_solver] use_gpu = yes against the stock CPU run:
its host loop then resolves the shim's GPU entry points
(set_model_initial_conditions_gpu / solve_model_odes_gpu) and keeps the state
in the shim's device rows.  The ToRORd cases carry the reference's extra data
(the stock transmural layers along x, and the z-layered adapter)."""
import os
import re
import subprocess
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
import make_golden as mg  # noqa: E402
import run_reference as rr  # noqa: E402

pytestmark = pytest.mark.gpu

SHIM = {m: os.path.join(REPO, "monoalg3d_c_b200", "shim", f"libmb_shim_{m}.so")
        for m in ("tt2006", "torord", "torord_endo")}


def _run(case, shim, gpu_host=False):
    """The reference binary on a fixture case (V dumped every 10 steps, the CG
    log of every step), with its stock plugins or with the shim; gpu_host runs
    the reference's GPU build with the cell model on the GPU."""
    with tempfile.TemporaryDirectory() as tmp:
        out_dir = os.path.join(tmp, "out")
        rc = dict(mg.reference_case(case), use_gpu=gpu_host)
        every = 10 if case.get("dt", 0.02) >= 0.02 else 100
        text = rr.ini_text(rc, tmp, out_dir, dumps_every=every)
        libs = rr.CUDA_LIBS if gpu_host else rr.LIBS
        if shim:
            lib = SHIM[case["model"]]
            stock_model = f"library_file={libs}/{rr.MODEL_LIBS[case['model']]}"
            stock_solver = f"library_file={libs}/libdefault_linear_system_solver.so"
            assert stock_model in text and stock_solver in text
            text = text.replace(stock_model, f"library_file={lib}").replace(stock_solver, f"library_file={lib}")
        ini = os.path.join(tmp, "case.ini")
        with open(ini, "w") as f:
            f.write(text)
        log = subprocess.run([rr.CUDA_BIN if gpu_host else rr.BIN, "-c", ini], capture_output=True, text=True, errors="replace",
                             timeout=600)
        assert log.returncode == 0, log.stdout[-2000:] + log.stderr[-2000:]
        its = [int(m.group(2)) for m in re.finditer(
            r"t = ([0-9.]+), Iterations = (\d+), Error Norm = ([0-9.eE+-]+)", log.stdout)]
        files = sorted((int(re.match(r"V_it_(\d+)\.bin$", f).group(1)), f)
                       for f in os.listdir(out_dir) if re.match(r"V_it_\d+\.bin$", f))
        V = np.stack([rr.read_bin(os.path.join(out_dir, f), case["nx"], case["ny"], case["nz"]) for _, f in files])
        return np.array(its), V, [c for c, _ in files]


def _compare(name, gpu_host):
    case = mg.CASES[name]
    model = case["model"]
    if not os.path.exists(SHIM[model]):
        pytest.skip("the shim is built only where the reference headers are mounted")
    its_ref, v_ref, counts_ref = _run(case, shim=False)
    its, v, counts = _run(case, shim=True, gpu_host=gpu_host)
    assert counts == counts_ref and len(its) == len(its_ref) and len(its) > 100
    assert np.array_equal(its, its_ref), f"{name}: CG iteration counts differ"
    ok = np.isfinite(v_ref)
    assert np.array_equal(ok, np.isfinite(v))
    err = np.abs(v[ok] - v_ref[ok])
    print(f"{name}: {len(its)} steps, max |dV| {err.max():.3e} mV")
    assert np.all(err <= 1e-8 * np.abs(v_ref[ok]) + 1e-9), f"{name}: max |dV| {err.max():.3e} mV"


@pytest.mark.skipif(not rr.available(), reason="the reference build (oracle/_ref) is not present")
@pytest.mark.parametrize("name", ["tt2006_cuboid", "torord_endo_cuboid", "tt2006_aniso_30",
                                  "torord_transmural_cuboid", "torord_fkatp_endo_euler"])
def test_reference_binary_with_shim(name):
    _compare(name, gpu_host=False)


@pytest.mark.skipif(not rr.cuda_available(), reason="the reference's GPU build (oracle/_ref/cuda) is not present")
@pytest.mark.parametrize("name", ["tt2006_cuboid", "torord_transmural_cuboid", "torord_rotating_transmural",
                                  "torord_fkatp_endo_euler"])
def test_reference_gpu_build_with_shim(name):
    _compare(name, gpu_host=True)

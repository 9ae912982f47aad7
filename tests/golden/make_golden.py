"""Generate the golden fixtures of the parity tests by running the reference
MonoAlg3D CPU path (FP64, OpenMP), built from its own sources into
oracle/_ref/ by oracle/ref/Makefile.

    python tests/golden/make_golden.py            # writes tests/golden/*.npz

Each case writes an ini file, runs oracle/_ref/bin/MonoAlg3D with the binary
V writer (save_as_text_or_binary, binary=true: centre, half sizes and V as
doubles per active cell), maps the cells to grid order by their centres and
stores V every `print_rate` steps plus the CG iterations and error of every
step from the solver log (and, for the ECG case, the reference's ecg.txt).  Runs only where the reference tree is mounted; the
fixtures are committed and the tests read only them.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")
BIN = os.path.join(REF, "bin", "MonoAlg3D")
LIBS = os.path.join(REF, "shared_libs")

# Each case: geometry (cells), model, assembly and simulation length.
CASES = {
    # the plain FP64 method on a small cuboid: TT2006, homogeneous sigma, Jacobi PCG 1e-16
    "tt2006_cuboid": dict(nx=32, ny=8, nz=2, model="tt2006", assembly="homogeneous", sim_ms=12.0),
    # ToRORd-fkatp endo/mid/epi library, no extra data (every cell ENDO)
    "torord_endo_cuboid": dict(nx=32, ny=8, nz=2, model="torord", assembly="homogeneous", sim_ms=12.0),
    # ToRORd with the reference's transmural extra data (45/25/30 % along x)
    "torord_transmural_cuboid": dict(nx=32, ny=8, nz=2, model="torord", assembly="homogeneous", sim_ms=12.0,
                                     extra_data=True),
    # anisotropic assembly, fibres along x (sigma_l / sigma_t)
    "tt2006_aniso_x": dict(nx=32, ny=8, nz=2, model="tt2006", assembly="anisotropic", fibre_deg=0.0, sim_ms=12.0),
    # anisotropic assembly, fibres at 30 degrees in the xy plane (cross terms)
    "tt2006_aniso_30": dict(nx=32, ny=8, nz=3, model="tt2006", assembly="anisotropic", fibre_deg=30.0, sim_ms=12.0),
    # pseudo-bidomain ECG (ecg_library/ecg.c) every 5 steps at three electrodes around the slab
    "tt2006_ecg": dict(nx=32, ny=16, nz=3, model="tt2006", assembly="homogeneous", sim_ms=30.0,
                       ecg=dict(leads=[[-500.0, 800.0, 150.0], [3700.0, 800.0, 150.0], [1600.0, -400.0, 150.0]],
                                sigma_b=1.0, calc_rate=5)),
}

DX = 100.0
DT = 0.02
PRINT_RATE = 50


def ini_text(case: dict, out_dir: str) -> str:
    nx, ny, nz = case["nx"], case["ny"], case["nz"]
    model_lib = {"tt2006": "libten_tusscher_2006.so", "torord": "libToRORd_fkatp_mixed_endo_mid_epi.so"}[case["model"]]
    if case["assembly"] == "homogeneous":
        assembly = ("main_function=homogeneous_sigma_assembly_matrix\n"
                    "sigma_x=0.00013\nsigma_y=0.00013\nsigma_z=0.00013\n")
    else:
        th = np.deg2rad(case["fibre_deg"])
        assembly = ("main_function=anisotropic_sigma_assembly_matrix\n"
                    "sigma_l=0.0002\nsigma_t=0.00005\nsigma_n=0.00005\n"
                    f"f=[{float(np.cos(th))!r},{float(np.sin(th))!r},0.0]\n")
    extra = ""
    if case.get("ecg"):
        e = case["ecg"]
        leads = "".join(f"lead{i + 1}={x!r},{y!r},{z!r}\n" for i, (x, y, z) in enumerate(e["leads"]))
        extra += ("[calc_ecg]\nmain_function=pseudo_bidomain\ninit_function=init_pseudo_bidomain\n"
                  f"end_function=end_pseudo_bidomain\ncalc_rate={e['calc_rate']}\n{leads}sigma_b={e['sigma_b']!r}\n"
                  f"use_gpu=no\nlibrary_file={LIBS}/libdefault_calc_ecg.so\n\n")
    if case.get("extra_data"):
        extra += ("[extra_data]\nmain_function=set_extra_data_mixed_torord_fkatp_epi_mid_endo\n"
                  f"library_file={LIBS}/libdefault_extra_data.so\n")
    return f"""[main]
num_threads=4
dt_pde={DT}
simulation_time={case['sim_ms']}
abort_on_no_activity=false
use_adaptivity=false

[update_monodomain]
main_function=update_monodomain_default
library_file={LIBS}/libdefault_update_monodomain.so

[save_result]
print_rate=1
output_dir={out_dir}
main_function=save_as_text_or_binary
binary=true
file_prefix=V
library_file={LIBS}/libdefault_save_mesh.so

[assembly_matrix]
init_function=set_initial_conditions_fvm
{assembly}library_file={LIBS}/libdefault_matrix_assembly.so

[linear_system_solver]
tolerance=1e-16
use_preconditioner=yes
max_iterations=200
library_file={LIBS}/libdefault_linear_system_solver.so
use_gpu=no
main_function=conjugate_gradient
init_function=init_conjugate_gradient
end_function=end_conjugate_gradient

[domain]
name=Cuboid Mesh
start_dx={DX}
start_dy={DX}
start_dz={DX}
side_length_x={nx * DX}
side_length_y={ny * DX}
side_length_z={nz * DX}
main_function=initialize_grid_with_cuboid_mesh
library_file={LIBS}/libdefault_domains.so

[ode_solver]
dt={DT}
use_gpu=no
gpu_id=0
library_file={LIBS}/{model_lib}

{extra}
[stim_plain]
start = 0.0
duration = 2.0
current = -53.0
x_limit = 500.0
main_function=stim_if_x_less_than
library_file={LIBS}/libdefault_stimuli.so
"""


def read_bin(path: str, nx: int, ny: int, nz: int) -> np.ndarray:
    rec = np.fromfile(path, dtype=np.float64).reshape(-1, 7)
    v = np.full(nx * ny * nz, np.nan)
    i = np.floor(rec[:, 0] / DX).astype(int)
    j = np.floor(rec[:, 1] / DX).astype(int)
    k = np.floor(rec[:, 2] / DX).astype(int)
    v[i + nx * (j + ny * k)] = rec[:, 6]
    return v


def run_case(name: str, case: dict) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        out_dir = os.path.join(tmp, "out")
        ini = os.path.join(tmp, f"{name}.ini")
        with open(ini, "w") as f:
            f.write(ini_text(case, out_dir))
        log = subprocess.run([BIN, "-c", ini, "-p", "1"], capture_output=True, text=True, check=True).stdout
        its, errs = [], []
        for m in re.finditer(r"t = ([0-9.]+), Iterations = (\d+), Error Norm = ([0-9.eE+-]+)", log):
            its.append(int(m.group(2)))
            errs.append(float(m.group(3)))
        counts = sorted(int(re.match(r"V_it_(\d+)\.bin$", f).group(1))
                        for f in os.listdir(out_dir) if re.match(r"V_it_\d+\.bin$", f))
        counts = [c for c in counts if c % PRINT_RATE == 0]
        V = np.stack([read_bin(os.path.join(out_dir, f"V_it_{c}.bin"), case["nx"], case["ny"], case["nz"])
                      for c in counts])
        res = dict(V=V, counts=np.array(counts), its=np.array(its), errors=np.array(errs),
                   config=json.dumps(dict(case, dx=DX, dt=DT, print_rate=PRINT_RATE)))
        if case.get("ecg"):
            # ecg.txt: time and one value per lead per line, "%lf" (ecg.c:286-306)
            rows = np.loadtxt(os.path.join(out_dir, "ecg.txt"), ndmin=2)
            res["ecg_t"] = rows[:, 0]
            res["ecg"] = rows[:, 1:]
    return res


def main(names=None):
    if not os.path.exists(BIN):
        sys.exit(f"{BIN} not built: run `make -C oracle/ref` first")
    for name in names or CASES:
        res = run_case(name, CASES[name])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **res)
        print(f"{name}: {len(res['its'])} steps, {len(res['counts'])} dumps, "
              f"mean CG its {res['its'].mean():.2f}")


if __name__ == "__main__":
    main(sys.argv[1:] or None)

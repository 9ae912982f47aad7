"""Runs the reference MonoAlg3D CPU path (oracle/_ref, built by oracle/ref/Makefile)
on a cuboid workload and reports its own timings.  Test and baseline
infrastructure only: the product never calls it.

cell-steps/s = active cells x loop steps / (Resolution Time - Total Write Time),
the reference's own clocks (monodomain_solver.c:936-946).
"""
from __future__ import annotations

import math
import os
import re
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "_ref")
BIN = os.path.join(REF, "bin", "MonoAlg3D")
LIBS = os.path.join(REF, "shared_libs")


def available() -> bool:
    return os.path.exists(BIN)


def physical_cores() -> int:
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return n
    except ImportError:
        pass
    return os.cpu_count() or 1


def ini_text(nx, ny, nz, dx, model, assembly, sim_ms, dt=0.02, threads=1, sigma=0.00013,
             sigma_l=0.0002, sigma_t=0.00005, f=(1.0, 0.0, 0.0), out_dir=None, print_rate=100000) -> str:
    model_lib = {"tt2006": "libten_tusscher_2006.so", "torord": "libToRORd_fkatp_mixed_endo_mid_epi.so"}[model]
    if assembly == "homogeneous":
        asm = f"main_function=homogeneous_sigma_assembly_matrix\nsigma_x={sigma}\nsigma_y={sigma}\nsigma_z={sigma}\n"
    else:
        asm = (f"main_function=anisotropic_sigma_assembly_matrix\nsigma_l={sigma_l}\nsigma_t={sigma_t}\n"
               f"sigma_n={sigma_t}\nf=[{f[0]!r},{f[1]!r},{f[2]!r}]\n")
    save = ""
    if out_dir:
        save = (f"[save_result]\nprint_rate={print_rate}\noutput_dir={out_dir}\nmain_function=save_as_text_or_binary\n"
                f"binary=true\nfile_prefix=V\nlibrary_file={LIBS}/libdefault_save_mesh.so\n")
    return f"""[main]
num_threads={threads}
dt_pde={dt}
simulation_time={sim_ms}
abort_on_no_activity=false
use_adaptivity=false

[update_monodomain]
main_function=update_monodomain_default
library_file={LIBS}/libdefault_update_monodomain.so

{save}
[assembly_matrix]
init_function=set_initial_conditions_fvm
{asm}library_file={LIBS}/libdefault_matrix_assembly.so

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
start_dx={dx}
start_dy={dx}
start_dz={dx}
side_length_x={nx * dx}
side_length_y={ny * dx}
side_length_z={nz * dx}
main_function=initialize_grid_with_cuboid_mesh
library_file={LIBS}/libdefault_domains.so

[ode_solver]
dt={dt}
use_gpu=no
gpu_id=0
library_file={LIBS}/{model_lib}

[stim_plain]
start = 0.0
duration = 2.0
current = -53.0
x_limit = 500.0
main_function=stim_if_x_less_than
library_file={LIBS}/libdefault_stimuli.so
"""


def loop_steps(final_time: float, dt: float) -> int:
    cur, n = 0.0, 0
    while cur - final_time <= dt:
        n += 1
        cur += dt
    return n


def run(nx, ny, nz, model, assembly, steps, dt=0.02, threads=None, dx=100.0, timeout=900, **kw) -> dict:
    """Runs about `steps` loop iterations and returns the timing summary."""
    threads = threads or physical_cores()
    sim_ms = max(0.0, (steps - 2) * dt)
    nsteps = loop_steps(sim_ms, dt)
    with tempfile.TemporaryDirectory() as tmp:
        ini = os.path.join(tmp, "bench.ini")
        with open(ini, "w") as f:
            f.write(ini_text(nx, ny, nz, dx, model, assembly, sim_ms, dt, threads, **kw))
        out = subprocess.run([BIN, "-c", ini], capture_output=True, text=True, timeout=timeout, check=True).stdout

    def grab(label):
        m = re.search(label + r": (\d+)", out)
        return int(m.group(1)) if m else 0

    res_us = grab("Resolution Time")
    write_us = grab("Total Write Time")
    cells = nx * ny * nz
    t = (res_us - write_us) * 1e-6
    return {"cells": cells, "steps": nsteps, "seconds": t, "threads": threads,
            "cell_steps_per_s": cells * nsteps / t if t > 0 else math.nan,
            "ode_s": grab("ODE Total Time") * 1e-6, "cg_s": grab("CG Total Time") * 1e-6,
            "cg_iterations": grab("CG Total Iterations")}

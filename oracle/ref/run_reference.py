"""Runs the reference MonoAlg3D CPU path (oracle/_ref, built by oracle/ref/Makefile)
on a structured tissue and reports its V dumps, CG log and its own timings.
TEST AND BASELINE INFRASTRUCTURE ONLY: the product never calls it.

A tissue is a `case` dict (see `ini_text`); `case_from_workload` derives one
from the benchmark workloads' keyword arguments without loading the product's
library.  Inputs the stock plugins cannot express go through the adapter
plugins of oracle/ref/adapters.c (libmb_adapters.so): a 3-D removed-cell
mask, fibres rotating linearly through the thickness, ToRORd cell types in
z-thirds, and V dumps every N steps.

cell-steps/s = active cells x loop steps / (Resolution Time - Total Write Time),
the reference's own clocks (monodomain_solver.c:936-946).
"""
from __future__ import annotations

import math
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "_ref")
BIN = os.path.join(REF, "bin", "MonoAlg3D")
LIBS = os.path.join(REF, "shared_libs")
# the reference's GPU build (Makefile.cuda): host loop with COMPILE_CUDA, GPU
# cell-model kernels, FP32 cuSPARSE / cuBLAS conjugate gradient
CUDA_BIN = os.path.join(REF, "cuda", "bin", "MonoAlg3D")
CUDA_LIBS = os.path.join(REF, "cuda", "shared_libs")

MODEL_LIBS = {"tt2006": "libten_tusscher_2006.so", "torord": "libToRORd_fkatp_mixed_endo_mid_epi.so",
              "torord_endo": "libToRORd_fkatp_endo.so"}


def available() -> bool:
    return os.path.exists(BIN) and os.path.exists(os.path.join(LIBS, "libmb_adapters.so"))


def cuda_available() -> bool:
    return os.path.exists(CUDA_BIN) and os.path.exists(os.path.join(CUDA_LIBS, "libmb_adapters.so"))


def physical_cores() -> int:
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return n
    except ImportError:
        pass
    return os.cpu_count() or 1


def loop_steps(final_time: float, dt: float) -> int:
    """Iterations of `while(cur_time - finalT <= dt_pde)` (monodomain_solver.c:616,908)."""
    cur, n = 0.0, 0
    while cur - final_time <= dt:
        n += 1
        cur += dt
    return n


def sim_ms_for_steps(steps: int, dt: float = 0.02) -> float:
    """A simulation_time whose loop runs `steps` iterations (T/dt + 2 for most T)."""
    return max(0.0, (steps - 2) * dt)


# ---- ini -----------------------------------------------------------------------

def _stim_section(i: int, s: dict) -> str:
    head = (f"[stim_{i}]\nstart = {float(s['start'])!r}\nduration = {float(s['duration'])!r}\n"
            f"current = {float(s['current'])!r}\n")
    if s.get("period"):
        head += f"period = {float(s['period'])!r}\n"
    if s["kind"] == "x_less_than":
        return head + (f"x_limit = {float(s['x_limit'])!r}\nmain_function=stim_if_x_less_than\n"
                       f"library_file={LIBS}/libdefault_stimuli.so\n")
    if s["kind"] == "x_y_limits":
        return head + (f"min_x = {float(s['min'][0])!r}\nmax_x = {float(s['max'][0])!r}\n"
                       f"min_y = {float(s['min'][1])!r}\nmax_y = {float(s['max'][1])!r}\n"
                       f"main_function=stim_x_y_limits\nlibrary_file={LIBS}/libdefault_stimuli.so\n")
    raise ValueError(f"stimulus kind {s['kind']!r} has no reference plugin here")


def ini_text(case: dict, work_dir: str, out_dir: str | None = None, dumps_every: int = 0,
             threads: int = 1) -> str:
    """The reference ini for a case.

    case keys: nx, ny, nz; dx (um, default 100); dt (ms, 0.02); sim_ms;
    model ("tt2006" | "torord"); assembly ("homogeneous" with sigma = 3
    values | "anisotropic" with sigma_l, sigma_t, sigma_n and either
    fibre_deg (one fibre in the xy plane) or fibre_rotate = (bottom_deg,
    top_deg)); mask (nx*ny*nz uint8, grid order, 0 = removed) or None;
    celltype (None = every ToRORd cell ENDO, "x_45_25_30" = the stock
    transmural extra data, "z_thirds" = the adapter's); stims (list of
    dicts: kind "x_less_than" | "x_y_limits", start, duration, current,
    x_limit | min, max); ecg (dict: leads, sigma_b, calc_rate) or None;
    use_gpu (the reference's GPU build: ODEs and CG on the GPU) and
    preconditioner (default True; the GPU CG has none);
    save_state (dict: output_dir, save_rate) and restore_state (dict:
    input_dir) for the reference's checkpoint plugins, or None; dt_ode (ms,
    default dt); adaptive (bool, forward-Euler model "torord_endo") with
    abs_tol, rel_tol; plugin_lib (a library file named in place of the stock
    cell model and linear solver: the reference-host plugins of
    monoalg3d_c_b200/shim)."""
    nx, ny, nz = case["nx"], case["ny"], case["nz"]
    dx = case.get("dx", 100.0)
    dt = case.get("dt", 0.02)
    if case["assembly"] == "homogeneous":
        sx, sy, sz = case.get("sigma", (0.00013,) * 3)
        asm = f"main_function=homogeneous_sigma_assembly_matrix\nsigma_x={sx!r}\nsigma_y={sy!r}\nsigma_z={sz!r}\n"
    else:
        asm = (f"main_function=anisotropic_sigma_assembly_matrix\nsigma_l={case['sigma_l']!r}\n"
               f"sigma_t={case['sigma_t']!r}\nsigma_n={case['sigma_n']!r}\n")
        if case.get("fibre_rotate") is not None:
            asm += "fibers_in_mesh=true\n"
        else:
            th = np.deg2rad(case.get("fibre_deg", 0.0))
            asm += f"f=[{float(np.cos(th))!r},{float(np.sin(th))!r},0.0]\n"
    dom_extra = ""
    if case.get("mask") is not None:
        mpath = os.path.join(work_dir, "mask.bin")
        np.ascontiguousarray(case["mask"], dtype=np.uint8).tofile(mpath)
        dom_extra += f"mask_file={mpath}\n"
    if case.get("fibre_rotate") is not None:
        b, t = case["fibre_rotate"]
        dom_extra += f"fibre_angle_bottom_deg={float(b)!r}\nfibre_angle_top_deg={float(t)!r}\n"
    if dom_extra:
        domain_fn, domain_lib = "initialize_grid_with_mb_cuboid", "libmb_adapters.so"
    else:
        domain_fn, domain_lib = "initialize_grid_with_cuboid_mesh", "libdefault_domains.so"
    extra = ""
    ct = case.get("celltype")
    if ct == "x_45_25_30":
        extra += ("[extra_data]\nmain_function=set_extra_data_mixed_torord_fkatp_epi_mid_endo\n"
                  f"library_file={LIBS}/libdefault_extra_data.so\n\n")
    elif ct == "z_thirds":
        extra += (f"[extra_data]\nmain_function=set_extra_data_mb_torord_z_layers\nstart_dz={dx!r}\n"
                  f"side_length_z={nz * dx!r}\nlibrary_file={LIBS}/libmb_adapters.so\n\n")
    elif ct is not None:
        raise ValueError(f"cell types {ct!r} have no reference plugin here")
    if case.get("ecg"):
        e = case["ecg"]
        leads = "".join(f"lead{i + 1}={x!r},{y!r},{z!r}\n" for i, (x, y, z) in enumerate(e["leads"]))
        extra += ("[calc_ecg]\nmain_function=pseudo_bidomain\ninit_function=init_pseudo_bidomain\n"
                  f"end_function=end_pseudo_bidomain\ncalc_rate={e['calc_rate']}\n{leads}sigma_b={e['sigma_b']!r}\n"
                  f"use_gpu=no\nlibrary_file={LIBS}/libdefault_calc_ecg.so\n\n")
    save = ""
    if out_dir:
        # print_rate 1 (the solver logs the CG of every step at the save
        # rate); the adapter writes the dumps every `dumps_every` steps
        save = (f"[save_result]\nprint_rate=1\noutput_dir={out_dir}\nmain_function=save_mb_v_every\n"
                f"every={dumps_every}\nlibrary_file={LIBS}/libmb_adapters.so\n")
    if case.get("save_state"):
        # the plain checkpoint plugin (save_state.c:16-150); save_rate 0 = at
        # the end of the run only
        ss = case["save_state"]
        save += (f"\n[save_state]\nsave_rate={int(ss.get('save_rate', 0))}\noutput_dir={ss['output_dir']}\n"
                 f"main_function=save_simulation_state\nlibrary_file={LIBS}/libdefault_save_state.so\n")
    if case.get("restore_state"):
        save += (f"\n[restore_state]\ninput_dir={case['restore_state']['input_dir']}\n"
                 f"main_function=restore_simulation_state\nlibrary_file={LIBS}/libdefault_restore_state.so\n")
    # ODE step: dt_ode (default dt); adaptive forward Euler with "adaptive"
    # (dt_ode None there = no dt line: the reference's min_dt of 1e-10)
    ode_dt = case.get("dt_ode", None if case.get("adaptive") else dt)
    ode_dt = "" if ode_dt is None else f"dt={ode_dt!r}\n"
    ode_adaptive = ""
    if case.get("adaptive"):
        ode_adaptive = (f"adaptive=true\nabstol={case.get('abs_tol', 1e-5)!r}\n"
                        f"reltol={case.get('rel_tol', 1e-5)!r}\n")
    stims = case.get("stims") or [dict(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)]
    stim_text = "\n".join(_stim_section(i, s) for i, s in enumerate(stims))
    text = f"""[main]
num_threads={threads}
dt_pde={dt}
simulation_time={case['sim_ms']}
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
use_preconditioner={'yes' if case.get('preconditioner', True) else 'no'}
max_iterations=200
library_file={LIBS}/libdefault_linear_system_solver.so
use_gpu={'yes' if case.get('use_gpu') else 'no'}
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
{dom_extra}main_function={domain_fn}
library_file={LIBS}/{domain_lib}

[ode_solver]
{ode_dt}{ode_adaptive}use_gpu={'yes' if case.get('use_gpu') else 'no'}
gpu_id=0
library_file={LIBS}/{MODEL_LIBS[case['model']]}

{extra}{stim_text}
"""
    if case.get("use_gpu"):
        text = text.replace(f"library_file={LIBS}/", f"library_file={CUDA_LIBS}/")
    if case.get("plugin_lib"):
        # another library in place of the stock cell model and linear solver
        # (the reference-host plugins of monoalg3d_c_b200/shim)
        libs = CUDA_LIBS if case.get("use_gpu") else LIBS
        for stock in (MODEL_LIBS[case["model"]], "libdefault_linear_system_solver.so"):
            text = text.replace(f"library_file={libs}/{stock}", f"library_file={case['plugin_lib']}")
    return text


# ---- workloads -----------------------------------------------------------------

def _attr(s, k, default=None):
    return s.get(k, default) if isinstance(s, dict) else getattr(s, k, default)


def case_from_workload(wl) -> dict:
    """The reference case of a benchmark workload (a Workload of
    monoalg3d_c_b200.workloads; read through its fields, without the
    product's library).  Raises ValueError for inputs no plugin expresses."""
    kw = wl.kwargs
    nx, ny, nz = wl.nx, wl.ny, wl.nz
    case = dict(nx=nx, ny=ny, nz=nz, dx=kw.get("dx", 100.0), dt=kw.get("dt_pde", 0.02),
                model=kw.get("model", "tt2006"), assembly=kw.get("assembly", "homogeneous"), sim_ms=wl.sim_ms)
    if kw.get("current_scale") is not None or kw.get("sigma_cell") is not None:
        raise ValueError("per-cell conductance scalings / conductivities have no reference plugin here")
    if case["assembly"] == "homogeneous":
        case["sigma"] = tuple(kw.get("sigma", (0.00013,) * 3))
    elif case["assembly"] == "anisotropic":
        case.update(sigma_l=kw["sigma_l"], sigma_t=kw["sigma_t"], sigma_n=kw.get("sigma_n", kw["sigma_t"]))
        th = kw.get("fibre_angle_z")
        th = np.zeros(nz) if th is None else np.asarray(th, dtype=np.float64)
        if np.all(th == th[0]):
            case["fibre_deg"] = float(np.rad2deg(th[0]))
        else:
            # theta_k = bottom + (top - bottom) (k + 1/2) / nz, in degrees
            deg = np.rad2deg(th)
            slope = (deg[-1] - deg[0]) / (nz - 1)
            bottom = deg[0] - 0.5 * slope
            top = bottom + slope * nz
            z = (np.arange(nz) + 0.5) / nz
            if not np.allclose(np.deg2rad(bottom + (top - bottom) * z), th, rtol=0, atol=1e-12):
                raise ValueError("fibre angles are not linear in z")
            case["fibre_rotate"] = (float(np.round(bottom, 9)), float(np.round(top, 9)))
    else:
        raise ValueError(f"assembly {case['assembly']!r} has no reference plugin here")
    if kw.get("active") is not None:
        case["mask"] = np.asarray(kw["active"], dtype=np.uint8)
    ct = kw.get("celltype")
    if ct is not None:
        ct = np.asarray(ct).reshape(nz, ny, nx)
        k = np.arange(nz)
        zt = np.minimum(2, (3 * k) // nz)
        if np.all(ct == zt[:, None, None]):
            case["celltype"] = "z_thirds"
        elif not np.all(ct == 0):
            raise ValueError("cell types other than z-thirds have no reference plugin here")
    case["stims"] = [dict(kind=_attr(s, "kind"), start=_attr(s, "start"), duration=_attr(s, "duration"),
                          current=_attr(s, "current"), period=_attr(s, "period", 0.0), x_limit=_attr(s, "x_limit"),
                          min=tuple(_attr(s, "min")), max=tuple(_attr(s, "max"))) for s in kw.get("stims", ())]
    return case


def sub_block(case: dict, nx: int, ny: int) -> dict:
    """The same case on the first nx x ny columns (full thickness): a
    bounded sample of a large tissue that keeps its z structure (cell
    types, fibre rotation)."""
    c = dict(case, nx=nx, ny=ny)
    if case.get("mask") is not None:
        c["mask"] = np.asarray(case["mask"]).reshape(case["nz"], case["ny"], case["nx"])[:, :ny, :nx].reshape(-1).copy()
    return c


# ---- runs ----------------------------------------------------------------------

def read_bin(path: str, nx: int, ny: int, nz: int, dx: float = 100.0) -> np.ndarray:
    """A binary V dump (7 doubles per active cell: centre, half sizes, V) in
    grid order; removed cells read NaN."""
    rec = np.fromfile(path, dtype=np.float64).reshape(-1, 7)
    v = np.full(nx * ny * nz, np.nan)
    i = np.floor(rec[:, 0] / dx).astype(int)
    j = np.floor(rec[:, 1] / dx).astype(int)
    k = np.floor(rec[:, 2] / dx).astype(int)
    v[i + nx * (j + ny * k)] = rec[:, 6]
    return v


def _grab(out: str, label: str) -> int:
    m = re.search(label + r": (\d+)", out)
    return int(m.group(1)) if m else 0


def run_case(case: dict, threads: int | None = None, dumps_every: int | None = None, timeout: float = 3600) -> dict:
    """Runs a case; returns the CG log of every step when dumps are asked
    (its, errors), the V dumps every `dumps_every` steps (counts, V: grid
    order), the ecg rows if asked, and the reference's own timings."""
    threads = threads or physical_cores()
    nx, ny, nz, dx = case["nx"], case["ny"], case["nz"], case.get("dx", 100.0)
    with tempfile.TemporaryDirectory() as tmp:
        out_dir = os.path.join(tmp, "out") if (dumps_every or case.get("ecg")) else None
        ini = os.path.join(tmp, "case.ini")
        with open(ini, "w") as f:
            f.write(ini_text(case, tmp, out_dir, dumps_every=dumps_every or 1000000000, threads=threads))
        binary = CUDA_BIN if case.get("use_gpu") else BIN
        # the GPU build prints the device UUID as raw bytes: decode leniently
        log = subprocess.run([binary, "-c", ini], capture_output=True, text=True, errors="replace", timeout=timeout,
                             check=True).stdout
        its, errs = [], []
        for m in re.finditer(r"t = ([0-9.]+), Iterations = (\d+), Error Norm = ([0-9.eE+-]+)", log):
            its.append(int(m.group(2)))
            errs.append(float(m.group(3)))
        res = dict(its=np.array(its), errors=np.array(errs))
        if dumps_every:
            counts = sorted(int(re.match(r"V_it_(\d+)\.bin$", f).group(1))
                            for f in os.listdir(out_dir) if re.match(r"V_it_\d+\.bin$", f))
            res["counts"] = np.array(counts)
            res["V"] = np.stack([read_bin(os.path.join(out_dir, f"V_it_{c}.bin"), nx, ny, nz, dx) for c in counts])
        if case.get("ecg"):
            rows = np.loadtxt(os.path.join(out_dir, "ecg.txt"), ndmin=2)
            res["ecg_t"] = rows[:, 0]
            res["ecg"] = rows[:, 1:]
    res_us, write_us = _grab(log, "Resolution Time"), _grab(log, "Total Write Time")
    cells = int(np.count_nonzero(case["mask"])) if case.get("mask") is not None else nx * ny * nz
    nsteps = loop_steps(case["sim_ms"], case.get("dt", 0.02))
    t = (res_us - write_us) * 1e-6
    res.update(cells=cells, steps=nsteps, seconds=t, threads=threads,
               cell_steps_per_s=cells * nsteps / t if t > 0 else math.nan,
               ode_s=_grab(log, "ODE Total Time") * 1e-6, cg_s=_grab(log, "CG Total Time") * 1e-6,
               cg_iterations=_grab(log, "CG Total Iterations"))
    return res


def time_case(case: dict, steps: int, threads: int | None = None, timeout: float = 3600) -> dict:
    """The case over `steps` loop iterations (a bounded sample in time), timed
    by the reference's own clocks."""
    c = dict(case, sim_ms=sim_ms_for_steps(steps, case.get("dt", 0.02)))
    r = run_case(c, threads=threads, timeout=timeout)
    r.pop("its", None)
    r.pop("errors", None)
    return r

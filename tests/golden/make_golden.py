"""Generate the golden fixtures of the parity tests by running the reference
MonoAlg3D CPU path (FP64, OpenMP), built from its own sources into
oracle/_ref/ by oracle/ref/Makefile, through oracle/ref/run_reference.py.

    python tests/golden/make_golden.py [case ...]     # writes tests/golden/<case>.npz

Each case runs the reference binary with V dumped every `PRINT_RATE` steps
(centre, half sizes and V as doubles per active cell, mapped to grid order by
the centres) and keeps V at those steps, the CG iterations and error of every
step from the solver log and, for the ECG case, the reference's ecg.txt.
Inputs the stock plugins cannot express (removed-cell masks, fibres rotating
through the thickness, z-layered ToRORd cell types) go through the adapter
plugins of oracle/ref/adapters.c.  torord_endo_steps holds one
forward-Euler step of the ToRORd_fkatp_endo library from many states (its
own solve_model_ode_cpu, called from the built plugin) and its CPU initial
state.  Runs only where the reference tree was built; the fixtures are
committed and the tests read only them.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
import run_reference as rr  # noqa: E402

DX = 100.0
DT = 0.02
PRINT_RATE = 50
SEED_MASK = 1001


def _philox_mask(n: int, phi: float) -> np.ndarray:
    """i.i.d. Bernoulli removal of a fraction phi, numpy's Philox keyed by the seed."""
    return (np.random.Generator(np.random.Philox(SEED_MASK)).random(n) >= phi).astype(np.uint8)


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
    # the precision configuration's tissue kind: ToRORd endo, fibres along x
    # (sigma_l 0.2, sigma_t 0.05 S/m), 20 % of the volumes removed (3-D mask)
    "torord_fibrosis_aniso": dict(nx=32, ny=16, nz=4, model="torord", assembly="anisotropic", fibre_deg=0.0,
                                  sigma_l=0.0002, sigma_t=0.00005, fibrosis=0.2, sim_ms=12.0),
    # the scale configuration's tissue kind: ToRORd in z-thirds endo / mid /
    # epi, fibres rotating from +60 to -60 degrees through the thickness
    # (sigma_l 0.2, sigma_t 0.04 S/m, 27-point rows)
    "torord_rotating_transmural": dict(nx=32, ny=16, nz=6, model="torord", assembly="anisotropic",
                                       fibre_rotate=(60.0, -60.0), sigma_l=0.0002, sigma_t=0.00004,
                                       z_thirds=True, sim_ms=12.0),
    # the forward-Euler library ToRORd_fkatp_endo, fixed step: dt_pde = dt_ode
    # = 2 us (its Euler step needs dt below twice the 1 us floor of the
    # release time constant; with num_steps > 1 the reference also sums the
    # stimulus of every sub-step into each of them)
    "torord_fkatp_endo_euler": dict(nx=32, ny=16, nz=3, model="torord_endo", assembly="homogeneous", dt=0.002,
                                    sim_ms=6.0, print_rate=500),
    # the same library with the adaptive Euler step as the stock examples run
    # it (adaptive = true, no ODE dt: min_dt 1e-10, max_dt = dt_pde)
    "torord_fkatp_endo_adaptive": dict(nx=32, ny=16, nz=3, model="torord_endo", assembly="homogeneous",
                                       adaptive=True, sim_ms=12.0),
}


def reference_case(case: dict) -> dict:
    """The run_reference case of a fixture case."""
    c = dict(nx=case["nx"], ny=case["ny"], nz=case["nz"], dx=DX, dt=case.get("dt", DT), model=case["model"],
             assembly=case["assembly"], sim_ms=case["sim_ms"])
    for k in ("dt_ode", "adaptive"):
        if k in case:
            c[k] = case[k]
    if case["assembly"] == "homogeneous":
        c["sigma"] = (0.00013, 0.00013, 0.00013)
    else:
        c.update(sigma_l=case.get("sigma_l", 0.0002), sigma_t=case.get("sigma_t", 0.00005))
        c["sigma_n"] = c["sigma_t"]
        if case.get("fibre_rotate"):
            c["fibre_rotate"] = tuple(case["fibre_rotate"])
        else:
            c["fibre_deg"] = case["fibre_deg"]
    if case.get("fibrosis"):
        c["mask"] = _philox_mask(case["nx"] * case["ny"] * case["nz"], case["fibrosis"])
    if case.get("extra_data"):
        c["celltype"] = "x_45_25_30"
    if case.get("z_thirds"):
        c["celltype"] = "z_thirds"
    if case.get("ecg"):
        c["ecg"] = case["ecg"]
    return c


def run_case(name: str, case: dict) -> dict:
    every = case.get("print_rate", PRINT_RATE)
    r = rr.run_case(reference_case(case), threads=4, dumps_every=every)
    res = dict(V=r["V"], counts=r["counts"], its=r["its"], errors=r["errors"],
               config=json.dumps(dict(case, dx=DX, dt=case.get("dt", DT), print_rate=every)))
    if case.get("ecg"):
        res["ecg_t"] = r["ecg_t"]
        res["ecg"] = r["ecg"]
    return res


def torord_endo_steps(n: int = 1024, dt: float = 0.002, seed: int = 11) -> dict:
    """One forward-Euler step of the ToRORd_fkatp_endo library
    (solve_model_ode_cpu, default_solvers.c:42-53) from n states: the
    library's CPU initial state with every state perturbed by up to +-5 %,
    V swept from -90 to +40 mV, every third cell stimulated (-53)."""
    import ctypes as C
    lib = C.CDLL(os.path.join(rr.LIBS, "libToRORd_fkatp_endo.so"))
    lib.solve_model_ode_cpu.argtypes = [C.c_double, C.POINTER(C.c_double), C.c_double]
    lib.set_model_initial_conditions_cpu.restype = None
    rng = np.random.Generator(np.random.Philox(seed))
    y0 = np.empty((n, 43))
    base = _endo_cpu_initial_state(lib)
    y0[:] = base * (1.0 + rng.uniform(-0.05, 0.05, size=(n, 43)))
    y0[:, 0] = np.linspace(-90.0, 40.0, n)
    stim = np.where(np.arange(n) % 3 == 0, -53.0, 0.0)
    y1 = y0.copy()
    for i in range(n):
        row = np.ascontiguousarray(y1[i])
        lib.solve_model_ode_cpu(dt, row.ctypes.data_as(C.POINTER(C.c_double)), stim[i])
        y1[i] = row
    return dict(y0=y0, y1=y1, stim=stim, dt=np.float64(dt), initial_state=base)


def _endo_cpu_initial_state(lib) -> np.ndarray:
    """The library's own CPU initial state: set_model_initial_conditions_cpu
    (ToRORd_fkatp_endo.c:4-78) on a one-cell struct ode_solver, of which the
    call reads original_num_cells and adaptive and sets sv (the leading
    members of ode_solver.h:49-70, mirrored up to sv, then padding)."""
    import ctypes as C

    class OdeSolverHead(C.Structure):
        _fields_ = [("handle", C.c_void_p), ("max_dt", C.c_double), ("min_dt", C.c_double),
                    ("auto_dt", C.c_bool), ("adaptive", C.c_bool), ("rel_tol", C.c_double),
                    ("abs_tol", C.c_double), ("num_cells_to_solve", C.c_size_t),
                    ("cells_to_solve", C.c_void_p), ("num_steps", C.c_uint32), ("gpu", C.c_bool),
                    ("gpu_id", C.c_int), ("original_num_cells", C.c_uint32),
                    ("sv", C.POINTER(C.c_double)), ("rest", C.c_char * 1024)]

    solver = OdeSolverHead()
    solver.original_num_cells = 1
    solver.adaptive = False
    lib.set_model_initial_conditions_cpu.argtypes = [C.POINTER(OdeSolverHead), C.c_void_p]
    lib.set_model_initial_conditions_cpu(C.byref(solver), None)
    return np.array([solver.sv[i] for i in range(43)])


def main(names=None, out_dir=HERE):
    if not rr.available():
        sys.exit(f"{rr.BIN} and the adapter plugins are not built: run `make -C oracle/ref` first")
    for name in names or list(CASES) + ["torord_endo_steps"]:
        if name == "torord_endo_steps":
            np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **torord_endo_steps())
            print(f"{name}: one Euler step of the endo library from 1024 states")
            continue
        res = run_case(name, CASES[name])
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **res)
        print(f"{name}: {len(res['its'])} steps, {len(res['counts'])} dumps, mean CG its {res['its'].mean():.2f}")


if __name__ == "__main__":
    main(sys.argv[1:] or None)

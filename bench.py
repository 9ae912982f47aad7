"""Benchmark of the operator-split monodomain step (cell-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config 1] [--impl ours|reference]

A step is one iteration of the reference time loop (ODE sub-steps, update_monodomain,
Jacobi-PCG to r.r <= 1e-16) on the whole tissue.  Default workload: the
precision configuration, a 200x200x50 slab (2M volumes, 20 % diffuse fibrosis,
1.6M active) with ToRORd endo cells and fibres along x, run in the
mixed-precision form; the plain FP64 GPU path is timed beside it and the
mixed/FP64 ratio and the V difference between the two are reported.

value  -- device time of K captured steps (CUDA events on the launching
          stream), inputs resident in HBM, max over ranks; whole-job cell-steps/s.
e2e    -- the same steps through the reference-host C-ABI call with host
          buffers: every step copies the stimulus currents host->device and
          V device->host (pinned host buffers).  The headline uses the
          pipelined call (mb_monodomain_step_host_async: the copies of a
          step run under the compute of the next ones, two buffer pairs);
          the synchronous call (mb_monodomain_step_host) is reported beside it.
Under torchrun each rank runs an independent replica (the path does not shard:
one GPU solves one tissue), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 4])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---- distributed plumbing (replicas) -----------------------------------------

def dist_init(args, backend: str = "nccl"):
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the
    launcher); the "gloo" backend runs the same plumbing on the CPU."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        import datetime
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- clocks during the timed region ---------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms while the
    timed steps run (the sampler is started just before and stopped just
    after them)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def wait_first(self, limit_s: float = 3.0):
        t0 = time.time()
        while self.proc and not self.rows and time.time() - t0 < limit_s:
            time.sleep(0.01)
        self.rows.clear()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if len(r) > 5 + q and "Active" in r[5 + q]
                          and "Not" not in r[5 + q]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# DRAM bytes per launch of the dominant kernel (dram__bytes_read.sum +
# dram__bytes_write.sum), keyed by workload and CG launch shape:
#   - from one ncu capture of the same workload and shape
#     (profiles/k_fcg_group_mixed_slab_200x200x50.md);
#   - per active cell and CG iteration, from a capture of a smaller case of
#     the same workload and shape (360x360x72, inputs larger than L2; the
#     interleaved sweep's traffic grows with the cells), scaled by the
#     launch's cells and iterations (profiles/k_fcg_group_mixed_slab_500x500x100.md).
# Keys: (workload, launch shape), else (workload, ("groups", sweep order)) --
# the four-cell-group shapes of one sweep order read and write the same data,
# so their DRAM traffic differs only by what L2 keeps between passes.
PROFILED_TRAFFIC = {("slab_200x200x50_torord_fibrosis20", 10): 145.5e6,
                    ("slab_200x200x50_torord_fibrosis20", 5): 177.3e6,
                    ("slab_200x200x50_torord_fibrosis20", ("groups", 0)): 177.3e6}
PROFILED_TRAFFIC_PER_CELL_ITERATION = {("slab_500x500x100_torord_rotating_fibres", 17): 58.83,
                                       ("slab_500x500x100_torord_rotating_fibres", ("groups", 1)): 58.83}
# Pipe utilisation of the mixed ODE kernel from one ncu capture of the same
# workload (profiles/k_torord_mixed_slab_200x200x50.md): XU = the MUFU pipe
# (ex2, lg2, rcp, rsqrt: the exp/log/divide-bound part), FMA = the FP32 pipe.
PROFILED_ODE_PIPES = {"slab_200x200x50_torord_fibrosis20": {"xu_pct": 46.8, "fma_pct": 32.8, "fp64_pct": 1.1,
                                                            "issue_active_pct": 53.7}}
FLAT_SHAPES_PER_ORDER = 12     # flat CG shapes per sweep order; the last 7 of each run four-cell groups


def traffic_key(cg_kernel: int):
    if 0 <= cg_kernel < 2 * FLAT_SHAPES_PER_ORDER and cg_kernel % FLAT_SHAPES_PER_ORDER >= 5:
        return ("groups", cg_kernel // FLAT_SHAPES_PER_ORDER)
    return cg_kernel


def measured_hbm():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# ---- algorithmic bytes (roofline numerators) --------------------------------------

def cg_bytes(prec: str, n_active: int, n_grid: int, its: float, refinements: float, masked: bool) -> float:
    """Bytes one CG solve must move at least: per iteration x, r, p each read and
    written once (Ap and z are not stored); plus the fused right-hand side and
    initial residual (read V*, read x, write r and p); 1 byte of mask per grid
    cell per iteration when cells are removed."""
    mask = n_grid * its if masked else 0.0
    if prec == "fp64":
        return n_active * 8.0 * (6 * its + 3) + mask
    # mixed: x in FP64 (16 B r+w), r and p in FP32 (8 + 8 B); every FP64
    # residual evaluation reads V* and x (16 B) and writes r, p (8 B)
    return n_active * (32.0 * its + 24.0 * max(refinements, 1.0)) + mask


def activation_error(wl, steps: int) -> dict:
    """Untimed: the workload in both precisions with activation (-30 mV)
    tracked on the device, first activation times compared after `steps`
    steps over the cells activated in both runs."""
    first = {}
    for prec in ("mixed", "fp64"):
        t = wl.tissue(precision=prec, track_activation=True)
        t.step(steps)
        t.sync()
        first[prec] = t.activation()["first"].astype(np.float64)
        t.close()
    a, b = first["mixed"], first["fp64"]
    both = (a >= 0) & (b >= 0)
    d = a[both] - b[both]
    return {"after_steps": steps, "cells_activated": int(both.sum()),
            "activated_in_one_run_only": int(((a >= 0) != (b >= 0)).sum()),
            "max_ms": float(np.abs(d).max()) if d.size else None,
            "rms_ms": float(np.sqrt(np.mean(d * d))) if d.size else None}


def ode_bytes(model: str, prec: str, n_active: int) -> float:
    """State read + written once per cell-step, plus V in and V* out."""
    per = {("tt2006", "fp64"): 18 * 8, ("tt2006", "mixed"): 5 * 8 + 13 * 4,
           ("torord", "fp64"): 42 * 8, ("torord", "mixed"): 8 * 8 + 34 * 4}[(model, prec)]
    return n_active * (2.0 * per + 16.0)


# ---- arms -------------------------------------------------------------------------

def run_tissue(wl, prec, steps, warmup, ws, gpu):
    t = wl.tissue(precision=prec)
    t.step(warmup)
    t.sync()
    barrier(ws)
    with ClockSampler(gpu) as clk:
        clk.wait_first()           # sampler running before the first timed step
        ms = t.time_steps(steps)
    t.sync()
    ms = allmax(ws, ms)
    prof = t.profile(3)        # phase times with events: ODE kernel, CG launch
    stats = t.step_stats(warmup, steps)
    return t, ms, prof, stats, clk.summary()


def cpu_baseline(wl, model, assembly):
    """The reference CPU path timed on this host: oracle/_ref (the reference's
    own build, OpenMP on all physical cores) when it is present, else the C
    restatement in oracle/ (kind "port", OpenMP)."""
    sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
    import run_reference
    if not run_reference.available():
        return cpu_baseline_port(wl, steps=3)
    r = run_reference.run(wl.nx, wl.ny, wl.nz, model, assembly, steps=6,
                          sigma_l=wl.kwargs.get("sigma_l", 0.0002), sigma_t=wl.kwargs.get("sigma_t", 0.00005))
    return {"value": r["cell_steps_per_s"], "unit": "cell-steps/s", "cores": r["threads"], "kind": "reference",
            "sample": f"reference MonoAlg3D CPU path (OpenMP, FP64, Jacobi-PCG 1e-16) on the {wl.nx}x{wl.ny}x{wl.nz} "
                      f"cuboid without removed cells, {r['steps']} loop steps, Resolution Time - Write Time"}


def cpu_baseline_port(wl, steps):
    """The oracle's C restatement of the reference loop (FP64, OpenMP) on the
    workload itself, `steps` loop steps after one untimed step."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    sim = oracle.Sim(wl.nx, wl.ny, wl.nz, **wl.kwargs)
    sim.step(1)
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    cells = wl.active_cells()
    sim.close()
    threads = int(os.environ.get("OMP_NUM_THREADS", "0")) or (os.cpu_count() or 1)
    return {"value": cells * steps / dt, "unit": "cell-steps/s", "cores": threads, "kind": "port",
            "sample": f"C restatement of the reference CPU path (oracle/, OpenMP, FP64) on the workload "
                      f"({cells} active cells), {steps} loop steps", "seconds": dt, "steps": steps}


def model_of(wl):
    return wl.kwargs.get("model", "tt2006")


def main():
    args = parse()
    # at least 3 untimed warm-up steps, whatever was asked; the line reports
    # the number taken
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_init(args)
    from monoalg3d_c_b200 import workloads
    wl = workloads.CONFIGS[args.config](args.scale)
    model = model_of(wl)
    assembly = wl.kwargs.get("assembly", "homogeneous")
    metric = "cell-steps/s (mixed precision)"
    if args.impl == "reference":
        if rank == 0:
            sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
            import run_reference
            if not run_reference.available():
                cb = cpu_baseline_port(wl, steps=max(args.steps // 100, 3))
                r = {"cell_steps_per_s": cb["value"], "seconds": cb["seconds"], "steps": cb["steps"],
                     "threads": cb["cores"], "kind": "port", "sample": cb["sample"]}
            else:
                r = run_reference.run(wl.nx, wl.ny, wl.nz, model, assembly, steps=max(args.steps // 100, 3),
                                      sigma_l=wl.kwargs.get("sigma_l", 0.0002),
                                      sigma_t=wl.kwargs.get("sigma_t", 0.00005))
            v = r["cell_steps_per_s"]
            sample = r.get("sample") or (f"reference MonoAlg3D CPU path (OpenMP, FP64) on the {wl.nx}x{wl.ny}x{wl.nz} "
                                         f"cuboid without removed cells, {r['steps']} loop steps")
            print(json.dumps({
                "impl": "reference", "metric": metric, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
                "steps": r["steps"], "warmup": 0, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": wl.name, "cells": wl.n},
                "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": r["threads"],
                                 "kind": r.get("kind", "reference"), "sample": sample},
                "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import ctypes
    n_active = wl.active_cells()
    masked = wl.kwargs.get("active") is not None
    t_mx, ms_mx, prof_mx, st_mx, clk_mx = run_tissue(wl, "mixed", args.steps, args.warmup, ws, local)
    t_64, ms_64, prof_64, st_64, clk_64 = run_tissue(wl, "fp64", args.steps, args.warmup, ws, local)

    # V difference of the two forms after the same steps
    v_mx, v_64 = t_mx.v(), t_64.v()
    ok = np.isfinite(v_64)
    dv = v_mx[ok] - v_64[ok]
    t_64.close()

    # end to end through the reference-host call with pinned host buffers
    import torch
    n_grid = wl.n
    # The host stimulus of these steps is the merged stimulus the workload's
    # protocol gives at their times.  Untimed steps first move the tissue past
    # every stimulus window the 2 x steps host-buffer steps would overlap, so
    # that value is zero -- and it is still copied to the device every step.
    dt = wl.kwargs.get("dt_pde", 0.02)
    t0 = t_mx.info()["cur_time"]
    t_end = t0 + 2 * args.steps * dt
    late = [s.start + s.duration for s in wl.kwargs.get("stims", ()) if s.start < t_end and s.start + s.duration > t0]
    if late:
        t_mx.step(int(np.ceil((max(late) - t0) / dt)) + 1)
    stim = torch.zeros(n_active, dtype=torch.float64, pin_memory=True)
    vout = torch.empty(n_grid, dtype=torch.float64, pin_memory=True)
    # the second buffer pair of the pipelined calls
    stim_b = stim.clone().pin_memory()
    vout_b = torch.empty(n_grid, dtype=torch.float64, pin_memory=True)
    barrier(ws)
    ms_e2e_sync = t_mx.time_steps_host(args.steps, ctypes.c_void_p(stim.data_ptr()),
                                       ctypes.c_void_p(vout.data_ptr()))
    ms_e2e_sync = allmax(ws, ms_e2e_sync)
    barrier(ws)
    ms_e2e = t_mx.time_steps_host_async(args.steps, stim.data_ptr(), stim_b.data_ptr(), vout.data_ptr(),
                                        vout_b.data_ptr())
    ms_e2e = allmax(ws, ms_e2e)
    tune = t_mx.tuning()
    t_mx_tuning = tune
    t_mx.close()
    # activation-time error of the mixed form (untimed, rank 0; 40 ms of the
    # workload; the 25 M-cell slab is left to the accuracy check module)
    if rank == 0 and wl.n <= 4_000_000:
        act_err = activation_error(wl, 2000)
    else:
        act_err = {"skipped": "run python -m monoalg3d_c_b200.accuracy_check for this workload"}

    cell_steps = n_active * args.steps * ws
    value = cell_steps / (ms_mx * 1e-3)
    fp64_value = cell_steps / (ms_64 * 1e-3)
    e2e = cell_steps / (ms_e2e * 1e-3)
    e2e_sync = cell_steps / (ms_e2e_sync * 1e-3)

    # roofline of the dominant kernel of the mixed step
    hbm, hbm_kind = measured_hbm()
    its = float(np.mean(st_mx["its"]))
    refs = float(np.mean(st_mx["refinements"]))
    cg_b = cg_bytes("mixed", n_active, n_grid, its, refs, masked)
    od_b = ode_bytes(model, "mixed", n_active)
    cg_kernel = t_mx_tuning["cg_kernel"]
    if prof_mx["cg_ms"] >= prof_mx["ode_ms"]:
        form = {100: "k_tcg, 2.5D tiled", 200: "k_rcg, resident tile columns"}.get(cg_kernel, "k_fcg, flat")
        name, b, dur = f"k_pcg<mixed> ({form} persistent Jacobi-PCG)", cg_b, prof_mx["cg_ms"]
    else:
        name, b, dur = f"k_{model}_mixed (Rush-Larsen ODE)", od_b, prof_mx["ode_ms"]
    achieved = b / (dur * 1e-3) / 1e9
    traffic, note = None, "algorithmic bytes / CUDA-event time"
    if name.startswith("k_pcg"):
        traffic = PROFILED_TRAFFIC.get((wl.name, cg_kernel), PROFILED_TRAFFIC.get((wl.name, traffic_key(cg_kernel))))
        if traffic is not None:
            note += "; traffic = DRAM bytes per launch measured by ncu (the solve's working set stays in L2)"
        per = PROFILED_TRAFFIC_PER_CELL_ITERATION.get(
            (wl.name, cg_kernel), PROFILED_TRAFFIC_PER_CELL_ITERATION.get((wl.name, traffic_key(cg_kernel))))
        if per is not None:
            traffic = per * n_active * its
            note += ("; traffic = DRAM bytes per cell-iteration measured by ncu on a 360x360x72 case of the "
                     "same kernel, times the launch's cells and iterations")
    roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic, "peak_kind": hbm_kind,
            "bytes_per_launch": b, "note": note}

    out = {
        "metric": metric, "value": value, "unit": "cell-steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mx / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded Philox fibrosis mask; workload shapes of the precision configuration)",
        "config": {"workload": wl.name, "cells": n_grid, "active_cells": n_active, "model": model,
                   "assembly": assembly, "dt_ms": 0.02, "cg_tolerance": 1e-16,
                   "l2": "inputs larger than L2 (state + vectors > 126 MB per step)",
                   "parallelism": f"replicas x{ws}"},
        "fp64": {"value": fp64_value, "ms_per_step": ms_64 / args.steps,
                 "cg_iterations_per_step": float(np.mean(st_64["its"])),
                 "ode_ms": prof_64["ode_ms"], "cg_ms": prof_64["cg_ms"], "clocks": clk_64},
        "mixed_over_fp64": value / fp64_value,
        "mixed": {"ode_ms": prof_mx["ode_ms"], "cg_ms": prof_mx["cg_ms"], "cg_iterations_per_step": its,
                  "fp64_residual_evaluations_per_step": refs, "ode_variant": tune["ode_variant"],
                  "cg_blocks": tune["cg_blocks"], "cg_kernel": tune["cg_kernel"]},
        "error_vs_fp64": {"v_rms_mv": float(np.sqrt(np.mean(dv ** 2))), "v_max_mv": float(np.max(np.abs(dv))),
                          "after_steps": args.warmup + args.steps + 3, "activation_ms": act_err},
        "roofline": roof,
        "ode_roofline": {"kernel": f"k_{model}_mixed (Rush-Larsen ODE)", "bound": "sfu/fp32 (MUFU) and hbm",
                         "achieved_hbm": od_b / (prof_mx["ode_ms"] * 1e-3) / 1e9, "peak_hbm": hbm, "unit": "GB/s",
                         "hbm_frac": od_b / (prof_mx["ode_ms"] * 1e-3) / 1e9 / hbm,
                         "pipes_ncu": PROFILED_ODE_PIPES.get(wl.name)},
        "kernels": {"ode_mixed": {"ms": prof_mx["ode_ms"], "bytes": od_b,
                                  "GBps": od_b / (prof_mx["ode_ms"] * 1e-3) / 1e9},
                    "cg_mixed": {"ms": prof_mx["cg_ms"], "bytes": cg_b,
                                 "GBps": cg_b / (prof_mx["cg_ms"] * 1e-3) / 1e9}},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": n_active * 8,
                "d2h_bytes_per_step": n_grid * 8,
                "call": "mb_monodomain_step_host_async (copies of every step overlapped with the next steps)",
                "synchronous": {"value": e2e_sync, "call": "mb_monodomain_step_host (copy in, step, copy out, wait)"}},
        "gpu_launches": 3 * args.steps,
        "clocks": clk_mx,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(wl, model, assembly)
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    if rank == 0:
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the operator-split monodomain step (cell-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--repeats R] [--config 4]
                    [--impl ours|reference|reference-gpu|reference-shim]

A step is one iteration of the reference time loop (ODE sub-steps,
update_monodomain, Jacobi-PCG to r.r <= 1e-16, clock) on the whole tissue.
Default workload: the scale configuration, a 500x500x100 slab (25 M volumes)
with ToRORd cells in transmural z-thirds and fibres rotating from +60 to -60
degrees through the thickness (27-point operator), run in the
mixed-precision form; the plain FP64 GPU path is timed beside it and the
mixed/FP64 ratio and the V difference between the two are reported.

value  -- device time of K captured steps (CUDA events on the launching
          stream), inputs resident in HBM, max over ranks; the K-step block
          is timed R times and the median block is reported (all blocks are
          listed); whole-job cell-steps/s.
e2e    -- the same steps through the reference-host C-ABI call with host
          buffers: every step copies the stimulus currents host->device and
          V device->host (pinned host buffers).  The headline uses the
          pipelined call (mb_monodomain_step_host_async: the copies of a
          step run under the compute of the next ones, two buffer pairs);
          the synchronous call (mb_monodomain_step_host) is reported beside it.
--impl reference times the reference's own CPU path (oracle/_ref, OpenMP on
the host's cores) on the same tissue -- adapter plugins express the
removed-cell mask, the rotating fibres and the z-layered cell types -- over a
bounded number of loop steps, by its own clocks; that process maps none of
this repository's CUDA code.  --impl reference-gpu times the reference's own
GPU build (oracle/_ref/cuda: its host loop, its GPU cell-model kernels and
its FP32 cuSPARSE/cuBLAS conjugate gradient) the same way, with the settings
of its GPU examples (no preconditioner, tolerance 1e-16, at most 200
iterations) -- the existing GPU code on the same GPU and tissue.
--impl reference-shim times the drop-in: the reference's CPU build with this
library's reference-host plugins (monoalg3d_c_b200/shim) as its cell model
and linear solver, on the same tissue, by its own clocks.
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
SMS = 148
MUFU_PER_SM_CLK = 16          # MUFU (ex2, lg2, rcp, rsqrt) results per SM per clock


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--config", type=int, default=4, choices=[0, 1, 2, 4])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu", "reference-shim"])
    ap.add_argument("--ref-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the untimed activation-time comparison")
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
    """nvidia-smi clocks and throttle reasons sampled every 20 ms while the
    timed steps run (started just before and stopped just after them)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None
        self.armed = False

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def wait_first(self, limit_s: float = 3.0):
        """Waits for the sampler's first row, then keeps only rows read
        from here on."""
        t0 = time.time()
        self.armed = True
        while self.proc and not self.rows and time.time() - t0 < limit_s:
            time.sleep(0.005)
        self.rows.clear()

    def _read(self):
        for line in self.proc.stdout:
            if self.armed:
                self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        self.armed = False
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if len(r) > 5 + q and "Active" in r[5 + q]
                          and "Not" not in r[5 + q]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---- profiled figures ----------------------------------------------------------------
#
# Figures from ncu captures, each keyed by the workload and the exact kernel
# it was captured on (the CG launch-shape id mb_monodomain_tuning reports, or
# the ODE kernel's name and variant); a figure is reported only when the
# bench's tuner picked that same kernel, else the field is null.
#   (workload, cg kernel id) -> DRAM bytes (dram__bytes_read.sum +
#   dram__bytes_write.sum) per active cell and CG iteration of one launch
PROFILED_CG_TRAFFIC = {
    # one-pass capture (dram__bytes_read.sum + dram__bytes_write.sum) of the
    # full 25 M-cell slab's second solve after tuning (the first to start
    # from the stored product), 15 iterations: k_zcg<1, 8, 3, 2, 2> 16.46 GB
    ("slab_500x500x100_torord_rotating_fibres", 307): 43.9,
}
#   (workload, "mixed" | "fp64", ode variant) -> pipe utilisation and MUFU
#   (XU pipe) warp instructions x 32 per cell-step of one launch
PROFILED_ODE = {
    # k_torord_mixed<0, 4> / k_torord_fp64<0, 3> on the 0.72-scale slab
    ("slab_500x500x100_torord_rotating_fibres", "mixed", 3): {
        "xu_pct": 48.9, "fma_pct": 34.7, "fp64_pct": 1.2, "dram_bytes_per_cell_step": 411.7,
        "mufu_per_cell_step": 227.0},
    ("slab_500x500x100_torord_rotating_fibres", "fp64", 2): {
        "fp64_pipe_pct": 17.2, "xu_pct": 4.4, "issue_active_pct": 20.6, "fp64_ops_per_cell_step": 3912.0,
        "mufu_per_cell_step": 248.3},
}


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured", float(d.get("sm_max_mhz", 1965.0))
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback", 1965.0


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


def ode_bytes(model: str, prec: str, n_active: int) -> float:
    """State read + written once per cell-step, plus V in and V* out."""
    per = {("tt2006", "fp64"): 18 * 8, ("tt2006", "mixed"): 5 * 8 + 13 * 4,
           ("torord", "fp64"): 42 * 8, ("torord", "mixed"): 8 * 8 + 34 * 4}[(model, prec)]
    return n_active * (2.0 * per + 16.0)


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


# ---- arms -------------------------------------------------------------------------

def run_tissue(wl, prec, steps, warmup, repeats, ws, gpu):
    """Creates the tissue, takes `warmup` untimed steps, then times `repeats`
    blocks of exactly `steps` steps (each bracketed by a barrier and device
    synchronisation); returns the per-block times (max over ranks)."""
    t = wl.tissue(precision=prec)
    t.step(warmup)
    t.sync()
    blocks = []
    with ClockSampler(gpu) as clk:
        clk.wait_first()           # sampler running before the first timed step
        for _ in range(repeats):
            barrier(ws)
            t.sync()
            ms = t.time_steps(steps)
            t.sync()
            blocks.append(allmax(ws, ms))
    prof = t.profile(3)        # phase times with events: ODE kernel, CG launch
    stats = t.step_stats(warmup, steps * repeats)
    return t, blocks, prof, stats, clk.summary()


def reference_case(wl):
    sys.path.insert(0, os.path.join(REPO, "oracle", "ref"))
    import run_reference
    return run_reference, run_reference.case_from_workload(wl)


def host_ram_bytes() -> int:
    try:
        import psutil
        return int(psutil.virtual_memory().available)
    except ImportError:
        return 0


# host memory the reference's octree grid takes per cell (measured: 1.8 KB
# per ToRORd cell with the 27-point anisotropic operator on the 25 M-cell
# slab, 2.3 KB on a 1.6 M-cell one), with a margin
REF_BYTES_PER_CELL = 2400


def reference_sample(rr, case, steps, threads=None, max_cells=None):
    """The reference CPU path on the case -- or, where the host cannot hold
    the reference's grid of the whole tissue (or max_cells is smaller), on
    its first columns at full thickness -- over `steps` loop steps from t = 0;
    its own clocks."""
    n = case["nx"] * case["ny"] * case["nz"]
    ram = host_ram_bytes()
    budget = ram // REF_BYTES_PER_CELL if ram else n
    if max_cells:
        budget = min(budget, max_cells)
    sub = case
    if n > budget:
        f = (budget / n) ** 0.5
        sx = max(4, int(case["nx"] * f) // 4 * 4)
        sy = max(4, int(case["ny"] * f) // 4 * 4)
        sub = rr.sub_block(case, sx, sy)
    r = rr.time_case(sub, steps, threads=threads)
    whole = sub is case
    what = (f"the whole {case['nx']}x{case['ny']}x{case['nz']} tissue" if whole else
            f"its first {sub['nx']}x{sub['ny']} columns at full thickness ({sub['nx']}x{sub['ny']}x{sub['nz']})")
    r["sample"] = (f"reference MonoAlg3D CPU path (oracle/_ref: OpenMP, FP64, Jacobi-PCG 1e-16; adapter plugins "
                   f"for mask / rotating fibres / z-layered cell types) on {what}, {r['steps']} loop steps from "
                   f"t = 0, Resolution Time - Total Write Time")
    r["whole_tissue"] = whole
    return r


def cpu_baseline(wl, rr_case):
    """The reference CPU path timed on this host on a bounded sample of the
    workload: its first columns at full thickness (at most a million cells),
    3 loop steps -- 10-30 s of CPU work; the C restatement in oracle/ (kind
    "port") where the reference build is absent."""
    rr, case = rr_case
    if not rr.available():
        return cpu_baseline_port(wl, steps=3)
    r = reference_sample(rr, case, 3, max_cells=1_000_000)
    return {"value": r["cell_steps_per_s"], "unit": "cell-steps/s", "cores": r["threads"], "kind": "reference",
            "sample": r["sample"]}


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
                      f"({cells} active cells), {steps} loop steps after one untimed step", "seconds": dt,
            "steps": steps}


def model_of(wl):
    return wl.kwargs.get("model", "tt2006")


def reference_arm(args, wl, metric):
    """--impl reference: the reference CPU path on the same workload.  Raises
    ValueError for inputs no reference plugin expresses."""
    rr, case = reference_case(wl)
    if rr.available():
        r = reference_sample(rr, case, max(args.ref_steps, 3))
        kind, sample, cells, warm = "reference", r["sample"], r["cells"], 0
    else:
        cb = cpu_baseline_port(wl, steps=max(args.ref_steps, 3))
        r = {"cell_steps_per_s": cb["value"], "seconds": cb["seconds"], "steps": cb["steps"],
             "threads": cb["cores"], "whole_tissue": True}
        kind, sample, cells, warm = "port", cb["sample"], wl.active_cells(), 1
    v = r["cell_steps_per_s"]
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
        "steps": r["steps"], "warmup": warm, "ms_per_step": 1e3 * r["seconds"] / r["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "cells": wl.n, "active_cells": wl.active_cells(),
                   "sampled_cells": int(cells), "same_tissue": bool(r["whole_tissue"])},
        "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": r["threads"], "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def reference_gpu_arm(args, wl, metric):
    """--impl reference-gpu: the reference's GPU build on the same tissue."""
    rr, case = reference_case(wl)
    if not rr.cuda_available():
        print(json.dumps({"impl": "reference_gpu", "unavailable": "the reference's GPU build (oracle/_ref/cuda) "
                                                                  "is not present"}))
        return
    gcase = dict(case, use_gpu=True, preconditioner=False)
    r = reference_sample(rr, gcase, max(args.ref_steps, 3))
    v = r["cell_steps_per_s"]
    print(json.dumps({
        "impl": "reference_gpu", "metric": metric, "value": v, "unit": "cell-steps/s", "n_gpus": 1,
        "steps": r["steps"], "ms_per_step": 1e3 * r["seconds"] / r["steps"], "higher_is_better": True,
        "dtype": "f64 cell model, f32 CG", "data": "synthetic",
        "config": {"workload": wl.name, "cells": wl.n, "active_cells": wl.active_cells(),
                   "sampled_cells": int(r["cells"]), "same_tissue": bool(r["whole_tissue"])},
        "settings": "reference GPU build (oracle/_ref/cuda, kernels for sm_100a): GPU cell model, FP32 "
                    "cuSPARSE/cuBLAS CG without preconditioner, tolerance 1e-16 on r.r, at most 200 iterations "
                    "(its GPU examples' settings); its own clocks, Resolution Time - Total Write Time",
        "phases_s": {"ode": r["ode_s"], "cg": r["cg_s"]},
        "cg_iterations_per_step": r["cg_iterations"] / r["steps"]}))


def reference_shim_arm(args, wl, metric):
    """--impl reference-shim: the drop-in as a MonoAlg3D user gets it -- the
    reference's own CPU build (its host loop, grid, assembly and
    update_monodomain) with this library's reference-host plugins
    (monoalg3d_c_b200/shim) named as its cell model and linear solver, on
    the same tissue; the reference's own clocks."""
    rr, case = reference_case(wl)
    shim = os.path.join(REPO, "monoalg3d_c_b200", "shim", f"libmb_shim_{case['model']}.so")
    if not rr.available() or not os.path.exists(shim):
        print(json.dumps({"impl": "reference_shim", "unavailable": "the reference build (oracle/_ref) or the "
                                                                   "shim plugins are not present"}))
        return
    r = reference_sample(rr, dict(case, plugin_lib=shim), max(args.ref_steps, 3))
    v = r["cell_steps_per_s"]
    print(json.dumps({
        "impl": "reference_shim", "metric": metric, "value": v, "unit": "cell-steps/s", "n_gpus": 1,
        "steps": r["steps"], "ms_per_step": 1e3 * r["seconds"] / r["steps"], "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "cells": wl.n, "active_cells": wl.active_cells(),
                   "sampled_cells": int(r["cells"]), "same_tissue": bool(r["whole_tissue"])},
        "settings": f"reference CPU build's host loop (oracle/_ref, {r['threads']} threads) with "
                    f"{os.path.basename(shim)} as its cell model and linear solver (FP64 cell model and "
                    "Jacobi-PCG on the GPU, tolerance 1e-16); its own clocks, Resolution Time - Total Write Time",
        "phases_s": {"ode": r["ode_s"], "cg": r["cg_s"]},
        "cg_iterations_per_step": r["cg_iterations"] / r["steps"]}))


def main():
    args = parse()
    # at least 3 untimed warm-up steps, whatever was asked; the line reports
    # the number taken
    args.warmup = max(args.warmup, 3)
    args.repeats = max(args.repeats, 1)
    metric = "cell-steps/s (mixed precision)"
    # the workload descriptions load none of the product's native code
    from monoalg3d_c_b200 import workloads
    if args.impl == "reference-gpu":
        if int(os.environ.get("RANK", "0")) == 0:
            reference_gpu_arm(args, workloads.CONFIGS[args.config](args.scale), metric)
        return
    if args.impl == "reference-shim":
        if int(os.environ.get("RANK", "0")) == 0:
            reference_shim_arm(args, workloads.CONFIGS[args.config](args.scale), metric)
        return
    if args.impl == "reference":
        # rank 0 alone runs the reference; no process group is needed
        if int(os.environ.get("RANK", "0")) == 0:
            try:
                reference_arm(args, workloads.CONFIGS[args.config](args.scale), metric)
            except ValueError as e:
                print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    ws, rank, local = dist_init(args)
    wl = workloads.CONFIGS[args.config](args.scale)

    import ctypes
    model = model_of(wl)
    assembly = wl.kwargs.get("assembly", "homogeneous")
    n_active = wl.active_cells()
    n_grid = wl.n
    masked = wl.kwargs.get("active") is not None
    t_mx, bl_mx, prof_mx, st_mx, clk_mx = run_tissue(wl, "mixed", args.steps, args.warmup, args.repeats, ws, local)
    t_64, bl_64, prof_64, st_64, clk_64 = run_tissue(wl, "fp64", args.steps, args.warmup, args.repeats, ws, local)
    ms_mx, ms_64 = statistics.median(bl_mx), statistics.median(bl_64)

    # V difference of the two forms after the same steps
    v_mx, v_64 = t_mx.v(), t_64.v()
    ok = np.isfinite(v_64)
    dv = v_mx[ok] - v_64[ok]
    tune_64 = t_64.tuning()
    t_64.close()

    # end to end through the reference-host call with pinned host buffers
    import torch
    # The host stimulus of these steps is the merged stimulus the workload's
    # protocol gives at their times.  Untimed steps first move the tissue past
    # every stimulus window the host-buffer steps would overlap, so that value
    # is zero -- and it is still copied to the device every step.
    dt = wl.kwargs.get("dt_pde", 0.02)
    t0 = t_mx.info()["cur_time"]
    t_end = t0 + (args.repeats + 1) * args.steps * dt
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
    e2e_blocks = []
    for _ in range(args.repeats):
        barrier(ws)
        ms = t_mx.time_steps_host_async(args.steps, stim.data_ptr(), stim_b.data_ptr(), vout.data_ptr(),
                                        vout_b.data_ptr())
        e2e_blocks.append(allmax(ws, ms))
    ms_e2e = statistics.median(e2e_blocks)
    tune = t_mx.tuning()
    t_mx.close()
    # activation-time error of the mixed form (untimed, rank 0): 1000 steps
    # (20 ms) of the workload in both precisions
    if args.no_accuracy:
        act_err = {"skipped": "--no-accuracy"}
    else:
        act_err = activation_error(wl, 1000) if rank == 0 else {"skipped": "rank 0 only"}

    cell_steps = n_active * args.steps * ws
    value = cell_steps / (ms_mx * 1e-3)
    fp64_value = cell_steps / (ms_64 * 1e-3)
    e2e = cell_steps / (ms_e2e * 1e-3)
    e2e_sync = cell_steps / (ms_e2e_sync * 1e-3)

    # roofline of the dominant kernel of the mixed step
    hbm, hbm_kind, sm_max = measured_peaks()
    its = float(np.mean(st_mx["its"]))
    refs = float(np.mean(st_mx["refinements"]))
    cg_b = cg_bytes("mixed", n_active, n_grid, its, refs, masked)
    od_b = ode_bytes(model, "mixed", n_active)
    cg_kernel = tune["cg_kernel"]
    if prof_mx["cg_ms"] >= prof_mx["ode_ms"]:
        name, b, dur = f"persistent Jacobi-PCG<mixed>, launch shape {cg_kernel}", cg_b, prof_mx["cg_ms"]
    else:
        name, b, dur = f"k_{model}_mixed (Rush-Larsen ODE)", od_b, prof_mx["ode_ms"]
    achieved = b / (dur * 1e-3) / 1e9
    traffic, note = None, "algorithmic bytes / CUDA-event time"
    per = PROFILED_CG_TRAFFIC.get((wl.name, cg_kernel)) if name.startswith("persistent") else None
    if per is not None:
        traffic = per * n_active * its
        note += "; traffic = ncu DRAM bytes per cell-iteration of this kernel, times the launch's cells and iterations"
    else:
        note += "; traffic null: no ncu capture of this exact kernel on this workload"
    roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic, "peak_kind": hbm_kind,
            "bytes_per_launch": b, "note": note}

    # ODE roofline: HBM fraction of the state traffic and, where an ncu capture
    # of the same kernel exists, the MUFU fraction from its instruction census
    mufu_peak = SMS * MUFU_PER_SM_CLK * sm_max * 1e6
    ode_roof = {"kernel": f"k_{model}_mixed (Rush-Larsen ODE)", "bound": "sfu/fp32 (MUFU) and hbm",
                "achieved_hbm": od_b / (prof_mx["ode_ms"] * 1e-3) / 1e9, "peak_hbm": hbm, "unit": "GB/s",
                "hbm_frac": od_b / (prof_mx["ode_ms"] * 1e-3) / 1e9 / hbm,
                "mufu_peak_per_s": mufu_peak}
    for prec, pr, tn in (("mixed", prof_mx, tune), ("fp64", prof_64, tune_64)):
        p = PROFILED_ODE.get((wl.name, prec, tn["ode_variant"]))
        cs = n_active / (pr["ode_ms"] * 1e-3)
        ode_roof[f"{prec}_cell_steps_per_s"] = cs
        if p:
            ode_roof[f"ncu_{prec}"] = dict(p, sfu_frac=p["mufu_per_cell_step"] * cs / mufu_peak)

    out = {
        "metric": metric, "value": value, "unit": "cell-steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mx / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded workload with the configuration's shapes and values)",
        "config": {"workload": wl.name, "cells": n_grid, "active_cells": n_active, "model": model,
                   "assembly": assembly, "dt_ms": 0.02, "cg_tolerance": 1e-16,
                   "l2": "inputs larger than L2 (state + vectors > 126 MB per step)",
                   "parallelism": f"replicas x{ws}", "repeats": args.repeats,
                   "timed_blocks_ms": bl_mx},
        "fp64": {"value": fp64_value, "ms_per_step": ms_64 / args.steps, "timed_blocks_ms": bl_64,
                 "cg_iterations_per_step": float(np.mean(st_64["its"])),
                 "ode_ms": prof_64["ode_ms"], "cg_ms": prof_64["cg_ms"], "cg_kernel": tune_64["cg_kernel"],
                 "ode_variant": tune_64["ode_variant"], "clocks": clk_64},
        "mixed_over_fp64": value / fp64_value,
        "mixed": {"ode_ms": prof_mx["ode_ms"], "cg_ms": prof_mx["cg_ms"], "cg_iterations_per_step": its,
                  "fp64_residual_evaluations_per_step": refs, "ode_variant": tune["ode_variant"],
                  "cg_blocks": tune["cg_blocks"], "cg_kernel": tune["cg_kernel"]},
        "error_vs_fp64": {"v_rms_mv": float(np.sqrt(np.mean(dv ** 2))), "v_max_mv": float(np.max(np.abs(dv))),
                          "after_steps": args.warmup + args.steps * args.repeats + 3, "activation_ms": act_err},
        "roofline": roof,
        "ode_roofline": ode_roof,
        "kernels": {"ode_mixed": {"ms": prof_mx["ode_ms"], "bytes": od_b,
                                  "GBps": od_b / (prof_mx["ode_ms"] * 1e-3) / 1e9},
                    "cg_mixed": {"ms": prof_mx["cg_ms"], "bytes": cg_b,
                                 "GBps": cg_b / (prof_mx["cg_ms"] * 1e-3) / 1e9}},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": n_active * 8,
                "d2h_bytes_per_step": n_grid * 8, "timed_blocks_ms": e2e_blocks,
                "call": "mb_monodomain_step_host_async (copies of every step overlapped with the next steps)",
                "synchronous": {"value": e2e_sync, "call": "mb_monodomain_step_host (copy in, step, copy out, wait)"}},
        "gpu_launches": 3 * args.steps * args.repeats,
        "clocks": clk_mx,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(wl, reference_case(wl))
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    if rank == 0:
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

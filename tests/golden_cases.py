"""Loading of the golden fixtures and construction of the matching tissues."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASE_NAMES = ["tt2006_cuboid", "torord_endo_cuboid", "torord_transmural_cuboid", "tt2006_aniso_x",
              "tt2006_aniso_30", "torord_fibrosis_aniso", "torord_rotating_transmural"]
# the forward-Euler library (ToRORd_fkatp_endo): fixed and adaptive step
ENDO_CASE_NAMES = ["torord_fkatp_endo_euler", "torord_fkatp_endo_adaptive"]
SEED_MASK = 1001


def load(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    out = {k: z[k] for k in z.files}
    out["config"] = json.loads(str(z["config"]))
    return out


def transmural_celltype(nx: int, ny: int, nz: int, dx: float) -> np.ndarray:
    """Cell types of set_extra_data_mixed_torord_fkatp_epi_mid_endo (extra_data.c:474-505):
    ENDO for x < 45 % of the side, MID up to 70 %, EPI beyond (the side is nx*dx
    for the power-of-two grids the fixtures use)."""
    side = nx * dx
    i = np.arange(nx)
    cx = (i + 0.5) * dx
    ct_x = np.where(cx < side * 0.45, 0, np.where(cx < side * 0.45 + side * 0.25, 1, 2)).astype(np.uint8)
    return np.broadcast_to(ct_x[None, None, :], (nz, ny, nx)).reshape(-1).copy()


def tissue_kwargs(cfg: dict) -> dict:
    from monoalg3d_c_b200 import Stim
    kw = dict(dx=cfg["dx"], dy=cfg["dx"], dz=cfg["dx"], dt_pde=cfg["dt"], model=cfg["model"],
              cg_tolerance=1e-16, cg_max_iterations=200, use_preconditioner=True,
              stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)])
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    if cfg["assembly"] == "homogeneous":
        kw.update(assembly="homogeneous", sigma=(0.00013, 0.00013, 0.00013))
    else:
        st = cfg.get("sigma_t", 0.00005)
        kw.update(assembly="anisotropic", sigma_l=cfg.get("sigma_l", 0.0002), sigma_t=st, sigma_n=st)
        if cfg.get("fibre_rotate"):
            # theta(k) = bottom + (top - bottom) (k + 1/2) / nz at the cell centres
            b, t = cfg["fibre_rotate"]
            kw["fibre_angle_z"] = np.deg2rad(b + (t - b) * ((np.arange(nz) + 0.5) / nz))
        else:
            kw["fibre_angle_z"] = np.full(nz, np.deg2rad(cfg["fibre_deg"]))
    if cfg.get("fibrosis"):
        kw["active"] = (np.random.Generator(np.random.Philox(SEED_MASK)).random(nx * ny * nz)
                        >= cfg["fibrosis"]).astype(np.uint8)
    if cfg.get("extra_data"):
        kw["celltype"] = transmural_celltype(nx, ny, nz, cfg["dx"])
    if cfg.get("dt_ode"):
        kw["dt_ode"] = cfg["dt_ode"]
    if cfg.get("adaptive"):
        kw["ode_adaptive"] = "cpu"     # the reference CPU build's adaptive Euler
    if cfg.get("z_thirds"):
        ct = np.minimum(2, (3 * np.arange(nz)) // nz).astype(np.uint8)
        kw["celltype"] = np.broadcast_to(ct[:, None, None], (nz, ny, nx)).reshape(-1).copy()
    return kw

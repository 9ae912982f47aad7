"""Loading of the golden fixtures and construction of the matching tissues."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASE_NAMES = ["tt2006_cuboid", "torord_endo_cuboid", "torord_transmural_cuboid", "tt2006_aniso_x",
              "tt2006_aniso_30"]


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
    if cfg["assembly"] == "homogeneous":
        kw.update(assembly="homogeneous", sigma=(0.00013, 0.00013, 0.00013))
    else:
        th = np.deg2rad(cfg["fibre_deg"])
        kw.update(assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00005, sigma_n=0.00005,
                  fibre_angle_z=np.full(cfg["nz"], th))
    if cfg.get("extra_data"):
        kw["celltype"] = transmural_celltype(cfg["nx"], cfg["ny"], cfg["nz"], cfg["dx"])
    return kw

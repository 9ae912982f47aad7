"""Seeded synthetic tissues with the shapes, sizes and value distributions of
the five benchmark configurations (there is no public dataset for this path).

All random draws use numpy's counter-based Philox generator keyed by a fixed
seed, in grid order (index i + nx*(j + ny*k)); the seeds are
fibrosis 1001, conductance scalings and instance sizes 2002, conductivity
field 3003, sensors and finite-difference directions 3004.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np

from .monodomain import Stim

# S/m -> mS/um as the reference ini expects (0.13 S/m -> sigma_x = 0.00013)
S_PER_M = 1e-3

SEED_FIBROSIS = 1001
SEED_SCALES = 2002
SEED_FIELD = 3003
SEED_SENSORS = 3004


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


def planar_stim(start: float = 0.0) -> Stim:
    """Planar stimulus of -53 uA/uF for 2 ms on volumes with x < 500 um."""
    return Stim(kind="x_less_than", start=start, duration=2.0, current=-53.0, x_limit=500.0)


@dataclass
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    kwargs: Dict = field(default_factory=dict)
    sim_ms: float = 0.0
    note: str = ""

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    def active_cells(self) -> int:
        a = self.kwargs.get("active")
        return self.n if a is None else int(np.count_nonzero(a))

    def tissue(self, **over):
        from .monodomain import Tissue
        kw = dict(self.kwargs)
        kw.update(over)
        return Tissue(self.nx, self.ny, self.nz, **kw)


def config0(scale: float = 1.0) -> Workload:
    """Plain method: 1.0 x 1.0 x 0.2 cm cuboid at 100 um (200k volumes), TT2006,
    isotropic 0.13 S/m, Jacobi PCG 1e-16, 100 ms."""
    nx, ny, nz = int(100 * scale), int(100 * scale), max(1, int(20 * scale))
    kw = dict(model="tt2006", precision="fp64", assembly="homogeneous",
              sigma=(0.13 * S_PER_M,) * 3, stims=[planar_stim()])
    return Workload("cuboid_100x100x20_tt2006", nx, ny, nz, kw, sim_ms=100.0)


def fibrosis_mask(n: int, phi: float, seed: int = SEED_FIBROSIS) -> np.ndarray:
    """i.i.d. Bernoulli removal of a fraction phi of the volumes."""
    return (rng(seed).random(n) >= phi).astype(np.uint8)


def config1(scale: float = 1.0) -> Workload:
    """Precision: 2 x 2 x 0.5 cm slab at 100 um (200x200x50 = 2M volumes), ToRORd
    endo, fibres along x with sigma_l 0.2 / sigma_t 0.05 S/m, 20 % diffuse
    fibrosis, 500 ms."""
    nx, ny, nz = int(200 * scale), int(200 * scale), max(1, int(50 * scale))
    mask = fibrosis_mask(nx * ny * nz, 0.2)
    kw = dict(model="torord", assembly="anisotropic", sigma_l=0.2 * S_PER_M, sigma_t=0.05 * S_PER_M,
              sigma_n=0.05 * S_PER_M, active=mask, stims=[planar_stim()])
    return Workload("slab_200x200x50_torord_fibrosis20", nx, ny, nz, kw, sim_ms=500.0)


def fibre_angles(nz: int, top_deg: float = -60.0, bottom_deg: float = 60.0) -> np.ndarray:
    """Fibre angle in the xy plane, linear in z from +60 deg (z = 0) to -60 deg (top),
    evaluated at the cell centres."""
    z = (np.arange(nz) + 0.5) / nz
    return np.deg2rad(bottom_deg + (top_deg - bottom_deg) * z)


def transmural_thirds(nx: int, ny: int, nz: int) -> np.ndarray:
    """ENDO / MID / EPI in z-thirds (0 / 1 / 2)."""
    k = np.arange(nz)
    ct_z = np.minimum(2, (3 * k) // nz).astype(np.uint8)
    return np.broadcast_to(ct_z[:, None, None], (nz, ny, nx)).reshape(-1).copy()


def config4(scale: float = 1.0) -> Workload:
    """Scale: 5 x 5 x 1 cm ventricular slab at 100 um (500x500x100 = 25M volumes),
    ToRORd with transmural thirds, fibres rotating +60 to -60 deg through the
    thickness (sigma_l 0.2, sigma_t 0.04 S/m, 19-point), S1 planar at t = 0 and
    an S2 quarter-domain stimulus at 320 ms, 1000 ms."""
    nx, ny, nz = int(500 * scale), int(500 * scale), max(1, int(100 * scale))
    s2 = Stim(kind="x_y_limits", start=320.0, duration=2.0, current=-53.0,
              min=(0.0, 0.0, 0.0), max=(nx * 100.0 / 2, ny * 100.0 / 2, 0.0))
    kw = dict(model="torord", assembly="anisotropic", sigma_l=0.2 * S_PER_M, sigma_t=0.04 * S_PER_M,
              sigma_n=0.04 * S_PER_M, fibre_angle_z=fibre_angles(nz),
              celltype=transmural_thirds(nx, ny, nz), stims=[planar_stim(), s2])
    return Workload("slab_500x500x100_torord_rotating_fibres", nx, ny, nz, kw, sim_ms=1000.0)


def config2_instances(scale: float = 1.0, n_cables: int = 128, n_sheets: int = 128):
    """The batching configuration's tissues: cables of length uniform 1-4 cm
    at 100 um (100-400 cells) and square sheets with side uniform 64-256
    cells, each with log-normal (sigma 0.2, median 1) scalings of gNa, gKr,
    gKs, gCaL and gK1.  Returns (sizes, scales)."""
    r = rng(SEED_SCALES)
    cable_len = np.rint(r.uniform(1.0, 4.0, n_cables) * 100.0 * scale).astype(int)
    sheet_side = np.rint(r.integers(64, 257, n_sheets) * scale).astype(int)
    sizes = [(max(2, int(c)), 1) for c in cable_len] + [(max(2, int(s)), max(2, int(s))) for s in sheet_side]
    scales = np.exp(0.2 * r.standard_normal((len(sizes), 5)))
    return sizes, scales


def config2(scale: float = 1.0):
    """Batching: 256 independent tissues (128 cables, 128 sheets), TT2006 with
    per-tissue scalings, isotropic 0.13 S/m, stimulus on the x = 0 edge,
    400 ms; outputs activation time and APD90 per cell.  Returns the batch's
    sizes, scales and Tissue keywords."""
    sizes, scales = config2_instances(scale)
    kw = dict(model="tt2006", assembly="homogeneous", sigma=(0.13 * S_PER_M,) * 3, track_activation=True)
    return sizes, scales, kw


def config2_workload(scale: float = 1.0) -> Workload:
    """The batching configuration as one atlas tissue (mb_batch_pack): the
    256 tissues side by side with removed cells between them."""
    from .batch import atlas
    sizes, scales, kw = config2(scale)
    W, H, x0, y0, akw = atlas(sizes, scales, Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0,
                                                  x_limit=100.0))
    kw = dict(kw)
    kw.update(akw)
    return Workload("batch_256_cables_and_sheets_tt2006", W, H, 1, kw, sim_ms=400.0,
                    note=f"{len(sizes)} tissues in a {W}x{H} atlas")


def gaussian_random_field(nx: int, ny: int, corr_cells: float, seed: int = SEED_FIELD) -> np.ndarray:
    """Unit-variance Gaussian random field with Gaussian covariance of
    correlation length corr_cells (in cells), made by filtering white noise
    in Fourier space (periodic), (ny, nx)."""
    w = rng(seed).standard_normal((ny, nx))
    kx = np.fft.fftfreq(nx)[None, :]
    ky = np.fft.fftfreq(ny)[:, None]
    # covariance exp(-r^2 / (2 l^2))  <->  spectral density ~ exp(-2 pi^2 l^2 k^2)
    filt = np.exp(-np.pi ** 2 * corr_cells ** 2 * (kx ** 2 + ky ** 2))
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    return (f - f.mean()) / f.std()


def config3(scale: float = 1.0):
    """Differentiation: 256 x 256 sheet at 100 um, TT2006, log sigma =
    log(0.13 S/m) + 0.3 g with g a Gaussian random field of correlation
    length 2 mm (20 cells); 64 sensor cells; V sampled every 1 ms over 200 ms;
    gradients at uniform sigma and gKr scaling 1, checkpoints every 50 steps.
    Returns a dict of the problem."""
    nx = ny = max(8, int(256 * scale))
    n = nx * ny
    g = gaussian_random_field(nx, ny, 20.0 * scale)
    sigma_true = 0.13 * S_PER_M * np.exp(0.3 * g.reshape(-1))
    sensors = rng(SEED_SENSORS).choice(n, size=64, replace=False)
    return dict(nx=nx, ny=ny, nsteps=int(round(200.0 / 0.02)), sample_every=50, checkpoint_every=50,
                sigma_true=sigma_true, sigma0=np.full(n, 0.13 * S_PER_M), gkr0=np.ones(n), sensors=sensors,
                stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=100.0)])


CONFIGS = {0: config0, 1: config1, 2: config2_workload, 4: config4}

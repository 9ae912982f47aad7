"""Pseudo-bidomain ECG on the device (ecg.cu; the reference's
pseudo_bidomain_cpu, ecg_library/ecg.c:204-307) against

  - the ecg.txt the reference MonoAlg3D wrote for the same run (golden
    fixture tt2006_ecg: 1502 steps, a record every 5 steps at three
    electrodes; the file holds six decimals), and
  - the oracle's restatement (oracle.pseudo_bidomain_ecg) evaluated on the
    device's own V at the recorded steps, with removed cells, in mixed
    precision and on the 27-point operator of rotating fibres.

Bars: within 1e-6 absolute of the reference's printed values; within 1e-10
relative (plus 1e-12 absolute) of the restatement on the same V."""
import os
import sys

import numpy as np
import pytest

import golden_cases as gc

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def test_ecg_matches_reference_ecg_txt():
    from monoalg3d_c_b200 import Tissue
    g = gc.load("tt2006_ecg")
    cfg = g["config"]
    e = cfg["ecg"]
    steps = len(g["its"])
    t = Tissue(cfg["nx"], cfg["ny"], cfg["nz"], **gc.tissue_kwargs(cfg), ecg_leads=e["leads"],
               ecg_rate=e["calc_rate"], ecg_sigma_b=e["sigma_b"], ecg_capacity=10000)
    t.step(steps)
    times, vals = t.ecg()
    t.close()
    ref = g["ecg"]
    assert vals.shape == ref.shape, (vals.shape, ref.shape)
    np.testing.assert_allclose(times, g["ecg_t"], rtol=0, atol=5e-7)
    err = np.abs(vals - ref)
    print(f"ECG vs reference ecg.txt: {len(times)} records, max |d| {err.max():.2e} (values up to {np.abs(ref).max():.2f})")
    assert err.max() <= 1e-6


CASES = {
    "masked_fp64": dict(nx=40, ny=24, nz=4, kw=dict(model="tt2006"), mask=0.2),
    "masked_mixed": dict(nx=40, ny=24, nz=4, kw=dict(model="torord", precision="mixed"), mask=0.15),
    "rotating_27pt": dict(nx=24, ny=16, nz=5, kw=dict(model="tt2006", assembly="anisotropic", sigma_l=0.0002,
                                                      sigma_t=0.00004,
                                                      fibre_angle_z=np.deg2rad(np.linspace(60, -60, 5)))),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_ecg_matches_restatement_on_device_v(name):
    from monoalg3d_c_b200 import Stim, Tissue
    c = CASES[name]
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    active = None
    if c.get("mask"):
        active = (np.random.default_rng(3).random(nx * ny * nz) >= c["mask"]).astype(np.uint8)
    leads = [[-300.0, 1200.0, 200.0], [nx * 100.0 + 400.0, 1000.0, 150.0], [2000.0, -500.0, 300.0],
             [1500.0, 1200.0, nz * 100.0 + 800.0]]
    rate = 7
    t = Tissue(nx, ny, nz, active=active, ecg_leads=leads, ecg_rate=rate, ecg_sigma_b=2.5, ecg_capacity=100,
               stims=[Stim(kind="x_less_than", start=0.0, duration=2.0, current=-53.0, x_limit=500.0)], **c["kw"])
    checked = 0
    for block in range(6):
        # records are taken at the start of the steps whose count is a
        # multiple of 7, of the V at that moment: after a multiple of 7 steps,
        # the next step records the V read now
        t.step(rate * 5)
        v = t.v()
        t.step(1)
        times, vals = t.ecg()
        got = vals[-1]
        want = oracle.pseudo_bidomain_ecg(v, nx, ny, nz, leads, 2.5, active=active)
        assert np.allclose(got, want, rtol=1e-10, atol=1e-12), f"{name} record {len(times) - 1}: {got} vs {want}"
        checked += 1
        t.step(rate - 1)
    assert checked == 6
    assert np.abs(vals).max() > 0
    t.close()

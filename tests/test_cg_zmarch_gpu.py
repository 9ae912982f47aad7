"""The z-march CG (cg_zmarch.cu: TMA-staged planes, tiles of 128 x W cells over
z chunks) on grids that exercise its tiling: several x tiles with a partial
last one, partial y tiles, several z chunks, and the rows' x / y face
classes at tile edges.  Every variant (forced through MB_CG_VARIANT) against
the CPU oracle after 60 steps of the rotating-fibre operator, ToRORd with
z-layered cell types: FP64 within 1e-8 relative with the oracle's CG
iteration count at every step; mixed precision within 2e-3 relative (+1 mV)
with iteration counts within one of the flat kernel's (the mixed table's
last three variants run the fused iteration: one stencil pass and one
reduction, r.z and r.r by recurrence)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

STEPS = 60
ZMARCH_VARIANTS = {"fp64": 7, "mixed": 10}


def _case():
    from monoalg3d_c_b200 import workloads
    nx, ny, nz = 264, 21, 7          # x tiles 128 + 128 + 8, y tiles partial for every W
    kw = dict(model="torord", assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00004, sigma_n=0.00004,
              fibre_angle_z=workloads.fibre_angles(nz), celltype=workloads.transmural_thirds(nx, ny, nz),
              stims=[workloads.planar_stim()])
    return nx, ny, nz, kw


def _run(precision, v, nx, ny, nz, kw):
    from monoalg3d_c_b200 import Tissue
    old = os.environ.get("MB_CG_VARIANT")
    try:
        os.environ["MB_CG_VARIANT"] = str(v)
        t = Tissue(nx, ny, nz, precision=precision, **kw)
    finally:
        if old is None:
            os.environ.pop("MB_CG_VARIANT", None)
        else:
            os.environ["MB_CG_VARIANT"] = old
    kernel = t.tuning()["cg_kernel"]
    t.step(STEPS)
    v_out = t.v()
    its = t.step_stats(0, STEPS)["its"]
    t.close()
    return kernel, v_out, its


@pytest.fixture(scope="module")
def reference():
    nx, ny, nz, kw = _case()
    o = oracle.Sim(nx, ny, nz, **kw)
    its = []
    for _ in range(STEPS):
        o.step(1)
        its.append(o.last_cg()[0])
    ref = o.v()
    o.close()
    return ref, np.array(its)


@pytest.mark.parametrize("z", range(ZMARCH_VARIANTS["fp64"]))
def test_zmarch_fp64_matches_oracle(reference, z):
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    ref, its_ref = reference
    nx, ny, nz, kw = _case()
    nf = cg_launch_shapes()
    kernel, got, its = _run("fp64", nf + 2 + z, nx, ny, nz, kw)
    assert kernel == 300 + z
    err = np.abs(got - ref)
    assert np.all(err <= 1e-8 * np.abs(ref) + 1e-9), f"variant {z}: max |dV| {err.max():.3e}"
    assert np.array_equal(its, its_ref), f"variant {z}: CG iterations {its} vs oracle {its_ref}"


@pytest.mark.parametrize("z", range(ZMARCH_VARIANTS["mixed"]))
def test_zmarch_mixed_matches_oracle_and_flat(reference, z):
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    ref, _ = reference
    nx, ny, nz, kw = _case()
    nf = cg_launch_shapes()
    _, _, its_flat = _run("mixed", 0, nx, ny, nz, kw)
    kernel, got, its = _run("mixed", nf + 2 + z, nx, ny, nz, kw)
    assert kernel == 300 + z
    err = np.abs(got - ref)
    assert np.all(err <= 2e-3 * (np.abs(ref) + 1.0)), f"variant {z}: max |dV| {err.max():.3e}"
    assert np.abs(its - its_flat).max() <= 1


@pytest.fixture(scope="module")
def reference_plain_cg():
    nx, ny, nz, kw = _case()
    o = oracle.Sim(nx, ny, nz, use_preconditioner=False, **kw)
    its = []
    for _ in range(STEPS):
        o.step(1)
        its.append(o.last_cg()[0])
    ref = o.v()
    o.close()
    return ref, np.array(its)


@pytest.mark.parametrize("precision,z", [("fp64", 0), ("fp64", 2), ("mixed", 1), ("mixed", 7), ("mixed", 8),
                                         ("mixed", 9)])
def test_zmarch_without_preconditioner(reference_plain_cg, precision, z):
    """The plain CG (use_preconditioner off: z = r, alpha = r.r / p.Ap, beta
    from r.r) through the ring and fused forms: FP64 within 1e-8 relative
    with the oracle's iteration counts, mixed within 2e-3 relative (+1 mV)
    with iteration counts within one of the flat mixed kernel's."""
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    ref, its_ref = reference_plain_cg
    nx, ny, nz, kw = _case()
    kw = dict(kw, use_preconditioner=False)
    nf = cg_launch_shapes()
    kernel, got, its = _run(precision, nf + 2 + z, nx, ny, nz, kw)
    assert kernel == 300 + z
    err = np.abs(got - ref)
    if precision == "fp64":
        assert np.all(err <= 1e-8 * np.abs(ref) + 1e-9), f"variant {z}: max |dV| {err.max():.3e}"
        assert np.array_equal(its, its_ref), f"variant {z}: CG iterations {its} vs oracle {its_ref}"
    else:
        _, _, its_flat = _run("mixed", 0, nx, ny, nz, kw)
        assert np.all(err <= 2e-3 * (np.abs(ref) + 1.0)), f"variant {z}: max |dV| {err.max():.3e}"
        assert np.abs(its - its_flat).max() <= 1


@pytest.mark.parametrize("shape", [(8, 1, 1), (12, 3, 2), (136, 9, 3), (260, 17, 1)])
def test_zmarch_small_and_ragged_grids(shape):
    """Edge shapes of the tiling: the narrowest grid the kernel takes (8 cells
    in x), one row, one plane, a last x tile of 4 or 8 cells, y tiles cut
    short for every W.  The ring and fused shapes against the oracle (FP64
    1e-8 relative with its iteration counts; mixed 2e-3 relative, +1 mV)."""
    from monoalg3d_c_b200 import workloads
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    nx, ny, nz = shape
    # fibres off the axes in every plane (one plane at 0 degrees would make
    # the operator the plain 7-point one, which the z-march does not take)
    kw = dict(model="torord", assembly="anisotropic", sigma_l=0.0002, sigma_t=0.00004, sigma_n=0.00004,
              fibre_angle_z=np.deg2rad(np.linspace(45.0, -30.0, nz)),
              celltype=workloads.transmural_thirds(nx, ny, nz), stims=[workloads.planar_stim()])
    o = oracle.Sim(nx, ny, nz, **kw)
    its_ref = []
    for _ in range(STEPS):
        o.step(1)
        its_ref.append(o.last_cg()[0])
    ref = o.v()
    o.close()
    nf = cg_launch_shapes()
    for precision, z in (("fp64", 0), ("fp64", 2), ("mixed", 1), ("mixed", 7), ("mixed", 9)):
        kernel, got, its = _run(precision, nf + 2 + z, nx, ny, nz, kw)
        assert kernel == 300 + z, f"{shape} {precision} variant {z} not used ({kernel})"
        err = np.abs(got - ref)
        if precision == "fp64":
            assert np.all(err <= 1e-8 * np.abs(ref) + 1e-9), f"{shape} variant {z}: max |dV| {err.max():.3e}"
            assert np.array_equal(its, np.array(its_ref)), f"{shape} variant {z}: CG iterations differ"
        else:
            assert np.all(err <= 2e-3 * (np.abs(ref) + 1.0)), f"{shape} mixed variant {z}: max |dV| {err.max():.3e}"


def test_fused_stored_product_and_outside_writes():
    """The fused solve starts from the product A x that its previous solve's
    last residual pass stored.  V written through the device pointer
    (mb_monodomain_device_v), behind the library's back, leaves that product
    stale: the next solve must still end on the stencil's own residual --
    the same V as a tissue whose V was set through mb_monodomain_set_v (which
    forgets the product) -- and only spend iterations on it."""
    from cuda.bindings import runtime as rt
    from monoalg3d_c_b200 import Tissue
    from monoalg3d_c_b200.monodomain import cg_launch_shapes
    nx, ny, nz, kw = _case()
    old = os.environ.get("MB_CG_VARIANT")
    try:
        os.environ["MB_CG_VARIANT"] = str(cg_launch_shapes() + 2 + 7)
        ta = Tissue(nx, ny, nz, precision="mixed", **kw)
        tb = Tissue(nx, ny, nz, precision="mixed", **kw)
    finally:
        if old is None:
            os.environ.pop("MB_CG_VARIANT", None)
        else:
            os.environ["MB_CG_VARIANT"] = old
    assert ta.tuning()["cg_kernel"] == 307 and tb.tuning()["cg_kernel"] == 307
    ta.step(20)
    tb.step(20)
    ta.sync()
    tb.sync()
    v = ta.v()
    vmod = v.copy()
    vmod[: nx * ny] += 5.0                        # the bottom plane 5 mV up
    tb.set_v(vmod)
    p, _ = ta.device_v()
    err, = rt.cudaMemcpy(p, vmod.ctypes.data, vmod.nbytes, rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    assert err == rt.cudaError_t.cudaSuccess
    ta.step(5)
    tb.step(5)
    va, vb = ta.v(), tb.v()
    sa, sb = ta.step_stats(20, 5), tb.step_stats(20, 5)
    ta.close()
    tb.close()
    assert np.all(sa["error"] <= 1e-16) and np.all(sb["error"] <= 1e-16)
    assert np.all(np.abs(va - vb) <= 1e-6 * (np.abs(vb) + 1.0)), f"max |dV| {np.abs(va - vb).max():.3e}"
    assert sa["its"][0] >= sb["its"][0]

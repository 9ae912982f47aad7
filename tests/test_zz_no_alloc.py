"""The allocation-free CSR conjugate gradient (mb_csr_conjugate_gradient_noalloc).

It serves callers that cannot allocate device memory while they run -- a host
framework that owns every device byte through its own pool, a real-time loop
that cannot take cudaMalloc's synchronisation, a plugin handed device buffers
by its host.  Such a caller passes its matrix, right-hand side and solution
already on the device; the entry point keeps its work vectors in a fixed
device array inside the library and allocates nothing.

This test (the test itself may allocate: it plays the caller's framework) puts
a symmetric positive definite system on the device with torch, solves it
twice in a row through the C ABI with the allocation-free entry point, and
checks each solution and iteration count against the allocating entry point
mb_csr_conjugate_gradient on the same system (same kernels, so the results
agree to rounding; the tolerance allows 1e-12 relative).  After one warm-up
call (the first call on a device places the library's fixed array there),
the device's free memory is the same before and after the two calls: they
allocate nothing.  It also checks that a system above the scratch limit is
rejected.  The file is named to be collected last and runs alone in a fresh
process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _laplacian_csr(nx, ny, shift):
    """5-point Laplacian plus shift*I on an nx x ny grid, CSR (SPD)."""
    n = nx * ny
    rows, cols, vals = [], [], []
    for j in range(ny):
        for i in range(nx):
            g = i + nx * j
            diag = shift
            for di, dj in ((-1, 0), (1, 0), (0, -1), (0, 1)):
                ii, jj = i + di, j + dj
                if 0 <= ii < nx and 0 <= jj < ny:
                    rows.append(g)
                    cols.append(ii + nx * jj)
                    vals.append(-1.0)
                    diag += 1.0
            rows.append(g)
            cols.append(g)
            vals.append(diag)
    rows = np.array(rows)
    order = np.lexsort((np.array(cols), rows))
    rows, cols, vals = rows[order], np.array(cols)[order], np.array(vals)[order]
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), cols.astype(np.int32), vals.astype(np.float64)


def test_noalloc_matches_allocating_solver_twice():
    import torch
    from monoalg3d_c_b200 import _lib, csr_conjugate_gradient

    torch.cuda.set_device(0)
    nx, ny = 96, 80
    row_ptr, col, val = _laplacian_csr(nx, ny, 0.07)
    n = nx * ny
    rng = np.random.default_rng(7)
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(row_ptr).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)

    def solve(d_b, d_x):
        its, err = C.c_uint32(), C.c_double()
        rc = _lib.lib.mb_csr_conjugate_gradient_noalloc(
            n, C.c_void_p(d_rp.data_ptr()), C.c_void_p(d_col.data_ptr()), C.c_void_p(d_val.data_ptr()),
            C.c_void_p(d_b.data_ptr()), C.c_void_p(d_x.data_ptr()), 1e-20, 500, 1, C.byref(its), C.byref(err),
            None)
        _lib.check(rc)
        return its.value, err.value

    # the references (the allocating solver) and every device buffer first
    cases = []
    for call in range(2):
        b = rng.standard_normal(n)
        x0 = rng.standard_normal(n) * 0.1
        ref = csr_conjugate_gradient(row_ptr, col, val, b, x0, tolerance=1e-20, max_iterations=500,
                                     use_preconditioner=True)
        cases.append((b, ref, torch.from_numpy(b).to(dev), torch.from_numpy(x0.copy()).to(dev)))
    warm_x = cases[0][3].clone()
    solve(cases[0][2], warm_x)         # places the fixed array on the device
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(0)[0]
    results = [solve(d_b, d_x) for (_, _, d_b, d_x) in cases]
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free_before, "the calls changed the device's free memory"

    for call, ((b, (x_ref, its_ref, err_ref), _, d_x), (its, err)) in enumerate(zip(cases, results)):
        x = d_x.cpu().numpy()
        assert its == its_ref, f"call {call}: {its} vs {its_ref} iterations"
        np.testing.assert_allclose(x, x_ref, rtol=1e-12, atol=1e-12 * np.abs(x_ref).max())
        assert err == pytest.approx(err_ref, rel=1e-9, abs=1e-30)
        # the solution really solves the system
        A = np.zeros(n)
        for r in range(n):
            A[r] = val[row_ptr[r]:row_ptr[r + 1]] @ x[col[row_ptr[r]:row_ptr[r + 1]]]
        assert np.linalg.norm(A - b) < 1e-8 * np.linalg.norm(b)


def test_noalloc_rejects_oversized_system():
    from monoalg3d_c_b200 import _lib
    its, err = C.c_uint32(), C.c_double()
    dummy = C.c_void_p(16)
    rc = _lib.lib.mb_csr_conjugate_gradient_noalloc((1 << 19) + 1, dummy, dummy, dummy, dummy, dummy, 1e-16, 10, 1,
                                                    C.byref(its), C.byref(err), None)
    assert rc == _lib.MB_ERR_ARG
    assert b"allocation-free limit" in _lib.lib.mb_last_error()

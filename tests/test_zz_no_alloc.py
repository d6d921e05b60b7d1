"""aphi_residuals_noalloc: residuals and backward errors without allocating.

For callers that cannot allocate device memory while they run (a serving
loop whose pool already owns the free device memory, a latency-critical path
that cannot take cudaFree's device-wide synchronization), the library offers
this one entry point with its scratch in a fixed device array. Checked here
through the C ABI against the allocating aphi_residuals on the same inputs,
on two calls in a row, plus its refusal of sizes beyond the array. Collected
last on purpose (file name), and self-contained: it builds its own problem,
so it passes alone in a fresh process as well as after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import aphi_b200 as ab

pytestmark = pytest.mark.gpu


def _call_noalloc(an, vals, x, b):
    batch, nrhs = b.shape[0], b.shape[1]
    out = np.zeros((batch, nrhs, 2))
    rc = ab.lib().aphi_residuals_noalloc(an._h, batch, nrhs, ab.dptr(vals), ab.dptr(x), ab.dptr(b),
                                         out.ctypes.data_as(C.POINTER(C.c_double)), None)
    return rc, out


def test_noalloc_residuals_match_the_allocating_entry_point(cuda):
    w = ab.Workload.cylinder(6)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, rhs = asm.refill(2 * np.pi * np.array([50.0, 1.0e5]))
    f = ab.Factor(an, batch=2)           # gives the analysis its device copy
    assert f.factorize(vals)
    rng = np.random.default_rng(11)
    b = torch.from_numpy(rng.normal(size=(2, 3, an.n)) + 1j * rng.normal(size=(2, 3, an.n))).cuda()
    b[:, 0] = rhs
    x = f.solve(b)
    for call in range(2):                # two calls in a row share the scratch array
        xc = x if call == 0 else (x * (1.0 + 1e-6)).contiguous()
        want = ab.residuals(an, vals, xc, b)
        rc, got = _call_noalloc(an, vals, xc, b)
        assert rc == ab.OK, ab.lib().aphi_last_error().decode()
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    assert got[:, 0, 1].max() < 1e-6      # the perturbed solution is still a near solution


def test_noalloc_refuses_sizes_beyond_its_array(cuda):
    w = ab.Workload.cylinder(4)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    f = ab.Factor(an)
    vals = torch.zeros((1, an.nnz), dtype=torch.complex128, device="cuda")
    v = torch.zeros((1, an.n), dtype=torch.complex128, device="cuda")
    out = np.zeros(2)
    rc = ab.lib().aphi_residuals_noalloc(an._h, 1, 1 << 22, ab.dptr(vals), ab.dptr(v), ab.dptr(v),
                                         out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == ab.ERR_BAD_SHAPE
    assert "fixed" in ab.lib().aphi_last_error().decode()
    del f

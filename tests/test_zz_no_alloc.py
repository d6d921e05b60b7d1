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
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc, got = _call_noalloc(an, vals, xc, b)
        assert rc == ab.OK, ab.lib().aphi_last_error().decode()
        if call == 1:                    # the first call may load the module that holds the array
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    assert got[:, 0, 1].max() < 1e-6      # the perturbed solution is still a near solution


def test_noalloc_needs_the_analysis_on_the_device(cuda):
    """An analysis that no factor has put on the device yet is refused: this
    entry point would have to allocate its device copy."""
    w = ab.Workload.cylinder(3)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    vals = torch.zeros((1, an.nnz), dtype=torch.complex128, device="cuda")
    v = torch.zeros((1, 1, an.n), dtype=torch.complex128, device="cuda")
    rc, _ = _call_noalloc(an, vals, v, v)
    assert rc == ab.ERR_INVALID
    assert "device copy" in ab.lib().aphi_last_error().decode()


def test_noalloc_at_the_size_limit_with_many_entries(cuda):
    """batch 64, one rhs each, on a diagonal pattern sized so that the scratch
    need is exactly the array's 2^20 doubles: the max|A| words of the 64
    entries sit right after the partial sums, at the array's end."""
    batch = 64
    nb = (2 ** 20 - 7 * batch) // (3 * batch)      # need = 3 nb batch + batch + 6 batch
    assert 3 * nb * batch + 7 * batch == 2 ** 20
    n = nb * 256 - 100
    rp = np.arange(n + 1, dtype=np.int32)
    ci = np.arange(n, dtype=np.int32)
    an = ab.Analysis(rp, ci, np.arange(n, dtype=np.int32))
    f = ab.Factor(an)                    # device copy of the analysis
    g = torch.Generator(device="cuda").manual_seed(5)
    vals = torch.randn((batch, n), dtype=torch.complex128, device="cuda", generator=g) + 3.0
    x = torch.randn((batch, 1, n), dtype=torch.complex128, device="cuda", generator=g)
    b = torch.randn((batch, 1, n), dtype=torch.complex128, device="cuda", generator=g)
    want = ab.residuals(an, vals, x, b)
    for _ in range(2):
        rc, got = _call_noalloc(an, vals, x, b)
        assert rc == ab.OK, ab.lib().aphi_last_error().decode()
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    del f


def test_noalloc_refuses_sizes_beyond_its_array(cuda):
    """Both refusals come before any launch, so the buffers handed in are
    never read: a scratch need beyond the array (300,000 unknowns x 400
    right-hand sides), and more systems than one launch's grid.y holds."""
    n = 300000
    an = ab.Analysis(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.arange(n, dtype=np.int32))
    f = ab.Factor(an)
    dummy = torch.zeros(2, dtype=torch.complex128, device="cuda")
    out = np.zeros(2)
    rc = ab.lib().aphi_residuals_noalloc(an._h, 1, 400, ab.dptr(dummy), ab.dptr(dummy), ab.dptr(dummy),
                                         out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == ab.ERR_BAD_SHAPE
    assert "fixed" in ab.lib().aphi_last_error().decode()
    w = ab.Workload.cylinder(4)
    an4 = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    f4 = ab.Factor(an4)
    rc = ab.lib().aphi_residuals_noalloc(an4._h, 1, 65536, ab.dptr(dummy), ab.dptr(dummy), ab.dptr(dummy),
                                         out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == ab.ERR_BAD_SHAPE
    assert "65535" in ab.lib().aphi_last_error().decode()
    del f, f4

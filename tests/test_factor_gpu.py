"""Device complex-symmetric LDL^T, solves and residuals against the reference.

The reference's known answers (tests/test_factorization.cpp) and its own
factorize_ldlt / solve_symmetric on the same matrices and the same analysis:
factor entries and solutions to <= 1e-10 relative, residuals <= 1e-12."""
import numpy as np
import pytest
import torch

import aphi_b200 as ab
from solvecheck import refined_solution, rel, spmv_extended  # noqa: F401

pytestmark = pytest.mark.gpu

SMALL_FRONTS = [96, 8]   # 8 sends every front past 8 rows through the blocked kernels


def opts(small_front):
    o = ab.default_analysis_options()
    o.small_front = small_front
    return o


def dense_to_upper(a):
    n = a.shape[0]
    rp, ci, v = [0], [], []
    for r in range(n):
        for c in range(r, n):
            if a[r, c] != 0 or r == c:
                ci.append(c)
                v.append(a[r, c])
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.complex128)


def factor_dense(a, perm=None, small_front=96, equil=0, floor=0.0):
    rp, ci, v = dense_to_upper(a)
    an = ab.Analysis(rp, ci, perm, options=opts(small_front))
    f = ab.Factor(an)
    vals = torch.from_numpy(v).cuda().unsqueeze(0)
    ok = f.factorize(vals, equil, floor)
    return an, f, ok, vals


def reconstruct(exp, n):
    L = np.eye(n, dtype=np.complex128)
    cp, ri, val = exp["col_ptr"], exp["row_index"], exp["value"]
    for j in range(n):
        for t in range(cp[j], cp[j + 1]):
            L[ri[t], j] = val[t]
    return L @ np.diag(exp["diagonal"]) @ L.T


@pytest.mark.parametrize("small_front", SMALL_FRONTS)
def test_two_by_two_by_hand(small_front, cuda):
    """tests/test_factorization.cpp:111-136: [[2,3],[3,5]] = L D L^T with
    L(1,0) = 3/2, D = [2, 1/2]."""
    a = np.array([[2, 3], [3, 5]], np.complex128)
    _, f, ok, _ = factor_dense(a, small_front=small_front)
    assert ok
    e = f.export()
    np.testing.assert_allclose(e["diagonal"], [2, 0.5], rtol=1e-15)
    np.testing.assert_allclose(e["value"], [1.5], rtol=1e-15)
    assert list(e["col_ptr"]) == [0, 1, 1] and list(e["row_index"]) == [1]


def test_zero_pivot_refused_at_column_one(cuda):
    """tests/test_factorization.cpp:253-276: [[0,1],[1,0]] is nonsingular but
    has no LDL^T without pivoting; the factorization stops at column 1."""
    a = np.array([[0, 1], [1, 0]], np.complex128)
    _, f, ok, _ = factor_dense(a)
    assert not ok
    assert f.stats[0]["ok"] == 0 and f.stats[0]["columns_done"] == 1
    with pytest.raises(ab.LogicError):
        f.solve(torch.zeros((1, 2), dtype=torch.complex128, device="cuda"))


@pytest.mark.parametrize("small_front", SMALL_FRONTS)
def test_no_conjugation(small_front, cuda):
    """A complex symmetric, non-Hermitian matrix reconstructs from L D L^T
    (transpose, not conjugate transpose) to 1e-14 (test_factorization.cpp:141-167)."""
    a = np.array([[4 + 1j, 1 - 2j, 0.5j], [1 - 2j, 3 - 1j, 2 + 0j], [0.5j, 2 + 0j, 5 + 3j]])
    _, f, ok, _ = factor_dense(a, small_front=small_front)
    assert ok
    r = reconstruct(f.export(), 3)
    assert np.abs(r - a).max() <= 1e-14 * np.abs(a).max()


def random_symmetric(rng, n, fill=0.12):
    a = np.zeros((n, n), np.complex128)
    for i in range(n):
        for j in range(i + 1, n):
            if rng.random() < fill:
                a[i, j] = a[j, i] = rng.normal() + 1j * rng.normal()
    a += np.diag(rng.normal(size=n) + 1j * rng.normal(size=n) + 6 * n + 0.5j * n)
    return a


@pytest.mark.parametrize("small_front", SMALL_FRONTS)
def test_random_patterns_match_reference(small_front, cuda, ref_or_skip):
    """Seeded random patterns n = 6..30 (the shape of test_factorization.cpp:169-213):
    under the reference's own AMD analysis, L and D agree with factorize_ldlt
    and L D L^T reconstructs P A P^T to 1e-12."""
    rng = np.random.default_rng(424242)
    for trial in range(30):
        n = int(rng.integers(6, 31))
        a = random_symmetric(rng, n)
        rp, ci, v = dense_to_upper(a)
        ref = ref_or_skip.RefProblem.from_pattern(rp, ci, ordering=2)
        ref.set_values(v)
        rf = ref.factorize()
        an_ref = ref.analysis()
        an = ab.Analysis(rp, ci, an_ref["perm"], an_ref["parent"], an_ref["col_count"], options=opts(small_front))
        f = ab.Factor(an)
        assert f.factorize(torch.from_numpy(v).cuda().unsqueeze(0), 0, 0.0)
        e = f.export()
        np.testing.assert_array_equal(e["col_ptr"], rf["col_ptr"])
        np.testing.assert_array_equal(e["row_index"], rf["row_index"])
        scale = np.abs(rf["value"]).max() if rf["value"].size else 1.0
        assert np.abs(e["value"] - rf["value"]).max(initial=0) <= 1e-12 * scale
        assert np.abs(e["diagonal"] - rf["diagonal"]).max() <= 1e-12 * np.abs(rf["diagonal"]).max()
        p = an_ref["perm"]
        pap = a[np.ix_(p, p)]
        assert np.abs(reconstruct(e, n) - pap).max() <= 1e-12 * np.abs(a).max()
        st = f.stats[0]
        assert st["nnz"] == rf["stats"]["nnz"]
        assert abs(st["largest_multiplier"] - rf["stats"]["largest_multiplier"]) <= 1e-12 * rf["stats"]["largest_multiplier"]
        assert abs(st["smallest_pivot"] - rf["stats"]["smallest_pivot"]) <= 1e-12 * rf["stats"]["smallest_pivot"]


OMEGAS = [2 * np.pi * 50.0, 2 * np.pi * 1e4, 2 * np.pi * 1e6]


@pytest.mark.parametrize("cells,small_front", [(6, 96), (6, 8), (8, 96), (12, 96), (12, 16), (16, 96)])
def test_cylinder_solve_symmetric_matches_reference(cells, small_front, cuda, ref_or_skip):
    """solve_symmetric on the cylinder-in-box (10 Ruiz iterations, the
    reference's AMD analysis) against the reference's solve_symmetric.

    Residual: <= 1e-12 relative. Solution: within 1e-10 of the reference's
    wherever the reference's own FP64 answer is that accurate; in general at
    least as accurate as the reference's, both measured against x*, the
    extended-precision refined solution. The system's conditioning grows with
    frequency: at 1 MHz the reference's own answer is ~1e-8 from x*, so no
    FP64 solver can agree with it to 1e-10 there."""
    w = ab.Workload.cylinder(cells)
    asm = ab.Assembly(ab.workload_arrays(w))
    ref = ref_or_skip.RefProblem.cylinder(cells)
    an_ref = ref.analysis()
    an = ab.Analysis(w.row_ptr, w.col_idx, an_ref["perm"], an_ref["parent"], an_ref["col_count"],
                     options=opts(small_front))
    for omega in OMEGAS:
        rv, rb = ref.refill(omega)
        xr, rep_r = ref.solve_symmetric(rb)
        ok, x, rep = ab.solve_symmetric(an, rv, rb)
        assert ok and rep_r["ok"]
        f = ab.Factor(an)
        assert f.factorize(torch.from_numpy(rv).cuda().unsqueeze(0))
        xs = refined_solution(f, w.row_ptr, w.col_idx, rv, rb, x)
        err_ref = rel(xr, xs)
        err_mine = rel(x, xs)
        assert err_mine <= max(1e-10, 2.0 * err_ref), (omega, err_mine, err_ref)
        assert rel(x, xr) <= 1e-10 + 3.0 * err_ref, (omega, rel(x, xr), err_ref)
        if err_ref <= 1e-11:
            assert rel(x, xr) <= 1e-10
        assert rep["residual"] <= 1e-12 and rep["backward_error"] <= 1e-16
        assert rep["factor_nnz"] == rep_r["factor_nnz"]
        assert abs(rep["equilibration_min"] / rep_r["equilibration_min"] - 1) < 1e-12
        assert abs(rep["equilibration_max"] / rep_r["equilibration_max"] - 1) < 1e-12
        assert abs(rep["smallest_pivot"] / rep_r["smallest_pivot"] - 1) < 1e-9
        assert abs(rep["largest_pivot"] / rep_r["largest_pivot"] - 1) < 1e-9
        # the device refill feeds the same numbers
        v, b = asm.refill(omega)
        assert np.array_equal(v[0].cpu().numpy(), rv)


def test_batched_factorization_equals_single(cuda, ref_or_skip):
    """Frequency batching: entries factorized together equal the same entries
    factorized alone, bit for bit (no reduction order depends on the batch)."""
    w = ab.Workload.cylinder(8)
    asm = ab.Assembly(ab.workload_arrays(w))
    an_ref = ref_or_skip.RefProblem.cylinder(8).analysis()
    an = ab.Analysis(w.row_ptr, w.col_idx, an_ref["perm"])
    om = np.geomspace(2 * np.pi * 50, 2 * np.pi * 1e6, 4)
    vals, rhs = asm.refill(om)
    fb = ab.Factor(an, batch=4)
    assert fb.factorize(vals)
    xb = fb.solve(rhs)
    for k in (0, 3):
        f1 = ab.Factor(an)
        assert f1.factorize(vals[k:k + 1])
        x1 = f1.solve(rhs[k:k + 1])
        assert bool((x1[0] == xb[k]).all())


def test_multiple_rhs_and_residuals(cuda, ref_or_skip):
    w = ab.Workload.cylinder(6)
    asm = ab.Assembly(ab.workload_arrays(w))
    an_ref = ref_or_skip.RefProblem.cylinder(6).analysis()
    an = ab.Analysis(w.row_ptr, w.col_idx, an_ref["perm"])
    vals, rhs = asm.refill(OMEGAS[1])
    f = ab.Factor(an)
    assert f.factorize(vals)
    rng = np.random.default_rng(7)
    b = torch.from_numpy(rng.normal(size=(1, 5, an.n)) + 1j * rng.normal(size=(1, 5, an.n))).cuda()
    x = f.solve(b)
    res = ab.residuals(an, vals, x, b)
    assert res.shape == (1, 5, 2)
    # Random right-hand sides on an ill-conditioned system: measured by the
    # backward error (the relative residual scales with the condition number).
    assert (res[..., 1] <= 1e-15).all(), res
    for k in range(5):
        xk = f.solve(b[:, k])
        assert bool((xk[0] == x[0, k]).all())     # each rhs independent of the others
    # ... and the physical right-hand side reaches the tight residual
    xp = f.solve(rhs)
    rp = ab.residuals(an, vals, xp, rhs)
    assert rp[0, 0, 0] <= 1e-12 and rp[0, 0, 1] <= 1e-16
    # more than 8 right-hand sides take several passes of the solve kernels
    b12 = torch.cat([b, b, b[:, :2]], dim=1)
    x12 = f.solve(b12)
    assert bool((x12[0, 5] == x[0, 0]).all()) and bool((x12[0, 11] == x[0, 1]).all())


def test_fp32_factor_with_fp64_refinement(cuda, ref_or_skip):
    """Mixed precision: FP32 factor, FP64 preconditioned-COCG refinement to the
    FP64 direct solve's residual level, and the automatic FP64 refactorization
    where the refinement stalls. Every solve of the sweep is at least as
    accurate as the reference's own (against x*), with relative residual
    <= 1e-12."""
    w = ab.Workload.cylinder(8)
    ref = ref_or_skip.RefProblem.cylinder(8)
    an_ref = ref.analysis()
    an = ab.Analysis(w.row_ptr, w.col_idx, an_ref["perm"])
    asm = ab.Assembly(ab.workload_arrays(w))
    om = np.array(OMEGAS)
    sweep = ab.SweepSolver(an, asm, len(om), "mixed", fp64_batch=2)
    x, vals, rhs, reports = sweep.solve(om)
    assert reports[0]["precision"] == "fp32"          # 50 Hz converges in FP32 + refinement
    res = ab.residuals(an, vals, x, rhs)
    assert (res[:, 0, 0] <= 1e-12).all(), res
    f64 = ab.Factor(an)
    for k, omega in enumerate(om):
        rv, rb = ref.refill(omega)
        xr, _ = ref.solve_symmetric(rb)
        assert f64.factorize(vals[k:k + 1])
        xs = refined_solution(f64, w.row_ptr, w.col_idx, rv, rb, xr)
        err_ref = rel(xr, xs)
        err = rel(x[k].cpu().numpy(), xs)
        assert err <= max(1e-10, 2.0 * err_ref), (omega, err, err_ref, reports[k])


def test_overlapped_fp64_entries_equal_sequential(cuda):
    """The second sweep of a mixed SweepSolver sends the frequencies it learned
    need FP64 straight to FP64; with overlap they are factorized on a side
    stream from a second thread while the FP32 entries refine. The answers
    must be the same bits as the sequential schedule's."""
    w = ab.Workload.cylinder(16)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    om = 2 * np.pi * np.geomspace(50.0, 1.0e6, 8)
    out = {}
    for overlap in (False, True):
        sw = ab.SweepSolver(an, asm, len(om), "mixed", fp64_batch=3, overlap=overlap)
        sw.solve(om)                       # learns the FP64 threshold
        x, vals, rhs, reps = sw.solve(om)  # predicted entries go to FP64 directly
        torch.cuda.synchronize()
        out[overlap] = (x.clone(), [r["precision"] for r in reps], [r["predicted_fp64"] for r in reps])
        sw.close()
    assert any(out[True][2]), "no entry was predicted to need FP64: the test does not exercise the overlap"
    assert out[True][1] == out[False][1]
    assert bool((out[True][0] == out[False][0]).all())
    res = ab.residuals(an, vals, out[True][0], rhs)
    assert (res[:, 0, 0] <= 1e-12).all()


def test_cocg_refinement_converges(cuda):
    """At 50 Hz and 20 kHz on 8^3 the FP32 factor preconditions COCG down to
    relative residual 1e-13, with the residual recomputed from x each step."""
    w = ab.Workload.cylinder(8)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, rhs = asm.refill(2 * np.pi * np.array([50.0, 2.0e4]))
    f = ab.Factor(an, precision=ab.PREC_FP32, batch=2)
    assert f.factorize(vals)
    x, iters, berr, ok = f.solve_refined(vals, rhs, tol=1e-16, rtol=1e-13, max_iters=40, krylov=True)
    res = ab.residuals(an, vals, x, rhs)
    assert ok and (res[:, 0, 0] <= 1e-13).all(), (iters, res)


@pytest.mark.parametrize("precision", [ab.PREC_FP64, ab.PREC_FP32])
def test_fused_solve_plans_equal_split_ones_bit_for_bit(precision, cuda):
    """The solves' fused plans (each triangle solved by the last CTA of the
    launch before it, handed over by an arrival counter) against the split
    plans (a launch per triangle): the same arithmetic in the same order, so
    the same bits, with 9 right-hand sides (two passes of the counters), a
    batch of 3, and twice in a row on one handle."""
    import os
    w = ab.Workload.cylinder(16)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, rhs = asm.refill(2 * np.pi * np.array([50.0, 1e4, 1e6]))
    g = torch.Generator(device="cuda").manual_seed(3)
    b = torch.randn(3, 9, an.n, 2, device="cuda", dtype=torch.float64, generator=g)
    b = torch.view_as_complex(b.contiguous())
    b[:, 0] = rhs
    saved = os.environ.get("APHI_SOLVE_SPLIT")
    xs = []
    try:
        for split in ("0", "1"):
            os.environ["APHI_SOLVE_SPLIT"] = split
            f = ab.Factor(an, precision=precision, batch=3)
            assert f.factorize(vals)
            for _ in range(2):
                xs.append(f.solve(b).cpu().numpy())
            f.close()
    finally:
        if saved is None:
            os.environ.pop("APHI_SOLVE_SPLIT", None)
        else:
            os.environ["APHI_SOLVE_SPLIT"] = saved
    assert np.isfinite(xs[0]).all()
    for x in xs[1:]:
        np.testing.assert_array_equal(x, xs[0])
    assert an.plan_stats(2).get("fwd_diag") is None and an.plan_stats(3).get("bwd_diag") is None


def test_prescaled_fp64_operand_matches_the_in_tile_scaling(cuda):
    """The FP64 trailing update on W = L D written once per panel group
    (k_dmma_scale) against the tile scaling its own A fragments
    (APHI_DMMA_PRESCALE=0): the same products, rounded in another kernel, so
    both solve to a relative residual <= 1e-12 and their solutions agree to
    1e-9 (cond(A) eps: the systems' conditioning grows with frequency); the
    scale launches run only in the first."""
    import os
    w = ab.Workload.cylinder(16)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    assert an.plan_stats(0).get("dmma_scale", (0, 0))[0] > 0
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, rhs = asm.refill(2 * np.pi * np.array([50.0, 1e4]))
    saved = os.environ.get("APHI_DMMA_PRESCALE")
    xs, launches = [], []
    try:
        for pre in ("1", "0"):
            os.environ["APHI_DMMA_PRESCALE"] = pre
            f = ab.Factor(an, precision=ab.PREC_FP64, batch=2)
            f.profile(True)
            assert f.factorize(vals)
            launches.append(f.profile_read().get("dmma_scale", (0, 0.0))[0])
            f.profile(False)
            x = f.solve(rhs)
            res = ab.residuals(an, vals, x, rhs)
            assert (res[:, 0, 0] <= 1e-12).all(), res
            xs.append(x.cpu().numpy())
            f.close()
    finally:
        if saved is None:
            os.environ.pop("APHI_DMMA_PRESCALE", None)
        else:
            os.environ["APHI_DMMA_PRESCALE"] = saved
    assert launches[0] > 0 and launches[1] == 0
    for k in range(2):
        assert np.linalg.norm(xs[0][k] - xs[1][k]) <= 1e-9 * np.linalg.norm(xs[1][k])


def test_factor_profile_counts_every_planned_launch(cuda):
    """aphi_factor_profile: one factorization with timing on records exactly
    the launches its plan holds, per kind, with positive durations. The
    operand-split launches run only for the two-piece split (the three-piece
    tile splits its operands itself)."""
    w = ab.Workload.cylinder(10)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, _ = asm.refill(2 * np.pi * np.array([50.0, 1e3]))
    for prec, plan, split in ((ab.PREC_FP64, 0, None), (ab.PREC_FP32, 1, 3), (ab.PREC_FP32, 1, 2)):
        f = ab.Factor(an, precision=prec, batch=2)
        if split:
            f.set_tc_split(split)
        f.profile(True)
        assert f.factorize(vals)
        got = f.profile_read()
        want = {k: v[0] for k, v in an.plan_stats(plan).items() if split != 3 or k != "tc_split"}
        if split == 2:
            assert want.get("tc_split", 0) > 0
        assert {k: v[0] for k, v in got.items()} == want
        assert all(ms > 0 for _, ms in got.values())
        f.profile(False)


def test_measured_peaks_are_plausible(cuda):
    p = ab.measure_peaks()
    assert 10 < p["fp64_dmma"] < 100 and 10 < p["fp64_dfma"] < 100
    assert 30 < p["fp32_ffma"] < 200
    assert 200 < p["tf32_tc_n64"] <= p["tf32_tc_n256"] * 1.05 < 3000


def test_set_batch_uses_part_of_the_capacity(cuda):
    """aphi_factor_set_batch: a factor made for 8 entries and used for 3
    (first use, and after a full batch) gives exactly the factorization and
    solutions of a factor made for 3."""
    w = ab.Workload.cylinder(6)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    vals, rhs = asm.refill(2 * np.pi * np.array([50.0, 7e2, 9e3]))
    ref = ab.Factor(an, batch=3)
    assert ref.factorize(vals)
    xr = ref.solve(rhs)
    big = ab.Factor(an, batch=8)
    for first in (True, False):
        if not first:
            v8, _ = asm.refill(2 * np.pi * np.geomspace(50, 1e4, 8))
            big.set_batch(8)
            assert big.factorize(v8)
        big.set_batch(3)
        assert big.factorize(vals)
        assert bool((big.solve(rhs) == xr).all())
    with pytest.raises(ab.InvalidArgument):
        big.set_batch(9)


def test_every_call_follows_the_callers_stream(cuda):
    """refill, factorize, solve and residuals all run on the stream they are
    given: on a non-blocking side stream, with no synchronization between
    the calls, the residual still sees the finished solution."""
    w = ab.Workload.cylinder(8)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    asm = ab.Assembly(ab.workload_arrays(w))
    f = ab.Factor(an, batch=16)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        vals, rhs = asm.refill(2 * np.pi * np.geomspace(50, 1e8, 16), stream=s)
        assert f.factorize(vals, stream=s)
        b = (torch.exp(1j * torch.linspace(0, 3, 8, dtype=torch.float64, device="cuda"))[None, :, None]
             * rhs[:, None, :]).contiguous()
        x = f.solve(b, stream=s)
        res = ab.residuals(an, vals, x, b, stream=s)
    assert (res[..., 0] <= 1e-12).all(), res[..., 0].max()

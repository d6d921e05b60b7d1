"""The C ABI library loads and exports every function include/aphi_b200.h
declares; the Python layer binds each one. CPU only (no compute calls)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import aphi_b200 as ab

HEADER = Path(__file__).resolve().parents[1] / "include" / "aphi_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(aphi_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) > 25
    lib = ctypes.CDLL(str(ab.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_layer_binds_every_declared_symbol():
    assert sorted(set(declared()) - set(ab.exported_symbols())) == []


def test_status_strings_and_errors_without_a_gpu():
    L = ab.lib()
    assert L.aphi_status_string(ab.ERR_PIVOT_FLOOR).decode() == "pivot at or below the floor"
    # a refused argument is reported, not thrown across the ABI
    rc = L.aphi_formulation_scales(ab.COND_ROW_SCALED, 0.0, None, None)
    assert rc == ab.ERR_BAD_SHAPE and "DC" in L.aphi_last_error().decode()


def test_analysis_matches_reference_etree_on_host():
    w = ab.Workload.cylinder(5)
    perm = ab.amd_ordering(w.row_ptr, w.col_idx)
    an = ab.Analysis(w.row_ptr, w.col_idx, perm)
    parent, cc = an.etree()
    assert (parent < 0).sum() == an.info["num_roots"]
    assert int(cc.sum()) == int(an.info["nnz_l"])
    # a wrong elimination tree handed in is refused as a logic error
    bad = parent.copy()
    bad[0] = -1 if bad[0] >= 0 else 1
    try:
        ab.Analysis(w.row_ptr, w.col_idx, perm, bad)
        raise AssertionError("expected a LogicError")
    except ab.LogicError:
        pass


def test_plan_stats_account_for_the_same_update_work():
    """Both factorization plans (DMMA / SIMT trailing tiles, tensor-core
    trailing tiles) do the same Schur-complement work, with the rest of a
    front updated once per group of 128-column panels (each panel before the
    group's last updates only the group's remaining columns): equal
    tiles and useful flops per kind, and as many useful flops as one update
    per panel would apply (the in-panel and trailing updates together carry
    the factorization's flops). Never more useful than executed; each plan
    uses only its own tile kind."""
    w = ab.Workload.cylinder(12)
    an = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx))
    assert an.info["max_width"] > 512   # fronts with several panel groups
    simt = an.plan_stats(0, flops=True)
    tc = an.plan_stats(1, flops=True)
    assert "update_tc" not in simt and "update_wide" not in tc
    assert simt["update_wide"][1] == tc["update_tc"][1]
    assert simt["update_wide"][2] == tc["update_tc"][2]
    # in-panel updates: 128 x 64 tiles on the trailing kernel in the FP64 plan,
    # 64 x 64 SIMT tiles in the tensor-core plan -- the same launches and work
    assert simt["update_panel"][0] == tc["update_panel"][0]
    assert simt["update_panel"][2] == tc["update_panel"][2]
    for st in (simt, tc):
        for kind, (_, _, useful, executed) in st.items():
            assert useful <= executed
    # the trailing and in-panel updates carry (almost) all of the factorization's flops
    total = simt["update_wide"][2] + simt["update_panel"][2]
    assert 0.9 * an.info["flops"] <= total <= 1.5 * an.info["flops"]
    # every trailing-update launch is preceded by its operand launch (W = L D in
    # the FP64 plan, the TF32 planes in the tensor-core plan), with one item per
    # 128 trailing rows of each front and no flops of its own
    assert simt["dmma_scale"][0] == simt["update_wide"][0]
    assert tc["tc_split"][0] == tc["update_tc"][0]
    assert simt["dmma_scale"][1] == tc["tc_split"][1]
    assert simt["dmma_scale"][2] == 0 and tc["tc_split"][2] == 0
    assert "tc_split" not in simt and "dmma_scale" not in tc


def _small_pattern():
    w = ab.Workload.cylinder(4)
    return w.row_ptr.copy(), w.col_idx.copy(), ab.amd_ordering(w.row_ptr, w.col_idx)


def test_analysis_refuses_malformed_input_on_host():
    """The analysis refuses what the reference refuses, before any device
    work: a perm that is not a permutation and malformed upper CSR
    (std::invalid_argument in the reference: InvalidArgument here), column
    counts that differ from the pattern's (std::logic_error: LogicError)."""
    rp, ci, perm = _small_pattern()
    n = rp.size - 1
    bad = perm.copy()
    bad[1] = bad[0]
    with pytest.raises(ab.InvalidArgument, match="permutation"):
        ab.Analysis(rp, ci, bad)
    bad = rp.copy()
    bad[5] = bad[4] - 1
    with pytest.raises(ab.InvalidArgument, match="row_ptr decreases"):
        ab.Analysis(bad, ci, perm)
    bad = ci.copy()
    bad[-1] = n
    with pytest.raises(ab.InvalidArgument, match="out of range"):
        ab.Analysis(rp, bad, perm)
    bad = ci.copy()
    r = 10                       # an entry below the diagonal in an upper pattern
    bad[rp[r]] = r - 1
    with pytest.raises(ab.InvalidArgument, match="below the diagonal"):
        ab.Analysis(rp, bad, perm)
    an = ab.Analysis(rp, ci, perm)
    parent, cc = an.etree()
    wrong = cc.copy()
    wrong[int(np.argmax(cc))] += 1
    with pytest.raises(ab.LogicError, match="column counts"):
        ab.Analysis(rp, ci, perm, parent, wrong)
    # the analysis of an empty pattern is empty, not an error
    empty = ab.Analysis(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert empty.info["n"] == 0 and empty.info["supernodes"] == 0


def test_orderings_edge_cases_on_host():
    """The reference's orderings through the C ABI: nothing to order at
    n = 0, a null argument refused, a diagonal-only pattern ordered as the
    reference orders isolated unknowns (AMD: degree buckets, last in first
    out; RCM: components by lowest vertex, then reversed)."""
    L = ab.lib()
    assert L.aphi_order_amd(0, None, None, None) == ab.OK
    assert L.aphi_order_rcm(0, None, None, None) == ab.OK
    assert L.aphi_order_rcm(3, None, None, None) == ab.ERR_INVALID
    assert L.aphi_order_amd(-1, None, None, None) == ab.ERR_INVALID
    n = 5
    rp = np.arange(n + 1, dtype=np.int32)
    ci = np.arange(n, dtype=np.int32)
    np.testing.assert_array_equal(ab.rcm_ordering(rp, ci), np.arange(n)[::-1])
    assert sorted(ab.amd_ordering(rp, ci).tolist()) == list(range(n))

"""Pins the C oracle (oracle/oracle.c) to the reference: against the golden
fixtures that tests/golden/make_golden.py wrote from the reference's own code,
and -- where oracle/_ref is built -- against the reference live. Also checks
the host-side pieces that must match the reference bit for bit: the workload
generator's pattern and the AMD restatement's permutation. CPU only."""
from pathlib import Path

import numpy as np
import pytest

import aphi_b200 as ab
import oraclelib as orc

GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    return dict(np.load(GOLD / name))


def test_element_blocks_bitwise_against_golden():
    g = load("element_blocks.npz")
    for c, (sigma, eps_r, mu_r, omega) in enumerate(g["cases"]):
        nu, alpha, beta = orc.coefficients(sigma, eps_r, mu_r, omega)
        for t in range(g["xyz"].shape[0]):
            aa, ap, pp = orc.element_blocks(g["xyz"][t], nu, alpha, beta)
            np.testing.assert_array_equal(aa, g["aa"][c, t])
            np.testing.assert_array_equal(ap, g["ap"][c, t])
            np.testing.assert_array_equal(pp, g["pp"][c, t])


def test_element_known_answer_unit_tet():
    """tests/test_element_matrix.cpp:101-134 (hand dot products {8,-4,0,4}/6)."""
    dots = np.array([[8, -4, -4, 4, 0, 4], [-4, 8, -4, -4, 4, 0], [-4, -4, 8, 0, -4, -4],
                     [4, -4, 0, 4, 0, 0], [0, 4, -4, 0, 4, 0], [4, 0, -4, 0, 0, 4]], float)
    aa, _, _ = orc.element_blocks(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float), 1.0, 0j, 0j)
    assert np.abs(aa - dots / 6).max() <= 1e-14


@pytest.mark.parametrize("cells", [4, 6])
def test_workload_and_amd_match_golden(cells):
    g = load(f"cylinder{cells}.npz")
    w = ab.Workload.cylinder(cells)
    np.testing.assert_array_equal(w.row_ptr, g["row_ptr"])
    np.testing.assert_array_equal(w.col_idx, g["col_idx"])
    np.testing.assert_array_equal(w.tet_idx, g["tet_idx"])
    np.testing.assert_array_equal(ab.amd_ordering(w.row_ptr, w.col_idx), g["perm"])
    an = ab.Analysis(w.row_ptr, w.col_idx, g["perm"])
    parent, cc = an.etree()
    np.testing.assert_array_equal(parent, g["parent"])
    np.testing.assert_array_equal(cc, g["col_count"])


@pytest.mark.parametrize("cells", [4, 6])
def test_refill_bitwise_against_golden(cells):
    g = load(f"cylinder{cells}.npz")
    arrays = ab.workload_arrays(ab.Workload.cylinder(cells))
    for k, om in enumerate(g["omegas"]):
        v, r = orc.refill(arrays, om)
        np.testing.assert_array_equal(v.view(np.float64), g["values"][k].view(np.float64))
        np.testing.assert_array_equal(r.view(np.float64), g["rhs"][k].view(np.float64))


@pytest.mark.parametrize("cells", [4, 6])
def test_solve_symmetric_against_golden(cells):
    g = load(f"cylinder{cells}.npz")
    for k in range(len(g["omegas"])):
        ok, x, rep = orc.solve_symmetric(g["row_ptr"], g["col_idx"], g["values"][k], g["rhs"][k], g["perm"],
                                         g["parent"], g["col_count"])
        assert ok
        np.testing.assert_array_equal(x.view(np.float64), g["x"][k].view(np.float64))
        np.testing.assert_array_equal(np.array(list(rep.values())), g["report"][k])
        d = orc.equilibration(g["row_ptr"], g["col_idx"], g["values"][k])
        np.testing.assert_array_equal(d, g["d"][k])


def test_factor_against_golden():
    g = load("cylinder4.npz")
    f = orc.factorize(g["row_ptr"], g["col_idx"], g["values"][0], g["perm"], g["parent"], g["col_count"])
    np.testing.assert_array_equal(f["col_ptr"], g["l_col_ptr"])
    np.testing.assert_array_equal(f["row_index"], g["l_row_index"])
    np.testing.assert_array_equal(f["value"].view(np.float64), g["l_value"].view(np.float64))
    np.testing.assert_array_equal(f["diagonal"].view(np.float64), g["l_diagonal"].view(np.float64))
    np.testing.assert_array_equal(np.array(list(f["stats"].values())), g["l_stats"])


def test_hand_and_random_matrices_against_golden():
    g = load("matrices.npz")
    for k in range(int(g["count"])):
        m = {key[len(f"m{k}_"):]: v for key, v in g.items() if key.startswith(f"m{k}_")}
        f = orc.factorize(m["row_ptr"], m["col_idx"], m["values"], m["perm"], m["parent"], m["col_count"])
        assert f["stats"]["ok"] == m["ok"] and f["stats"]["columns_done"] == m["columns_done"]
        np.testing.assert_array_equal(f["row_index"], m["l_row_index"])
        if m["ok"]:
            np.testing.assert_array_equal(f["value"], m["l_value"])
            np.testing.assert_array_equal(f["diagonal"], m["l_diagonal"])
            ok, x, _ = orc.solve_symmetric(m["row_ptr"], m["col_idx"], m["values"], m["b"], m["perm"],
                                           m["parent"], m["col_count"], equil_iters=0)
            np.testing.assert_array_equal(x, m["x"])
    # tests/test_factorization.cpp:111-136 by hand: L(1,0) = 3/2, D = [2, 1/2]
    assert g["m0_l_value"][0] == 1.5 and list(g["m0_l_diagonal"]) == [2, 0.5]
    # :253-276: [[0,1],[1,0]] refused at column 1
    assert int(g["m1_ok"]) == 0 and int(g["m1_columns_done"]) == 1


def test_oracle_detects_a_planted_mistake():
    """A mistake planted in the oracle's input (one conjugated value) is
    caught: the factor of the modified matrix no longer matches."""
    g = load("matrices.npz")
    v = g["m2_values"].copy()
    v[1] = np.conj(v[1])
    f = orc.factorize(g["m2_row_ptr"], g["m2_col_idx"], v, g["m2_perm"], g["m2_parent"], g["m2_col_count"])
    assert not np.array_equal(f["value"], g["m2_l_value"])


@pytest.mark.parametrize("cells", [3, 8])
def test_oracle_against_live_reference(cells, ref_or_skip):
    r = ref_or_skip.RefProblem.cylinder(cells)
    arrays = ab.workload_arrays(ab.Workload.cylinder(cells))
    an = r.analysis()
    rp, ci = r.pattern()
    for om in 2 * np.pi * np.array([50.0, 2.0e5]):
        rv, rr = r.refill(om)
        v, b = orc.refill(arrays, om)
        np.testing.assert_array_equal(v, rv)
        np.testing.assert_array_equal(b, rr)
        xr, repr_ = r.solve_symmetric(rr)
        ok, x, rep = orc.solve_symmetric(rp, ci, rv, rr, an["perm"], an["parent"], an["col_count"])
        assert ok
        np.testing.assert_array_equal(x, xr)
        assert rep["backward_error"] == repr_["backward_error"]

"""The synthetic workload generators (cylinder-in-box, torus with a cut port)
against the reference's own host pipeline
(build_topology, bind_to_mesh with the tree-cotree gauge, build_dof_map,
local_dofs, build_sparsity): bit-exact, so the GPU path is fed the same
matrices the reference assembles. CPU only."""
import numpy as np
import pytest

import aphi_b200 as ab


@pytest.mark.parametrize("cells", [3, 4, 6, 8, 10])
def test_cylinder_matches_reference_pipeline(cells, ref_or_skip):
    w = ab.Workload.cylinder(cells)
    r = ref_or_skip.RefProblem.cylinder(cells, ordering=-1)
    assert (w.num_nodes, w.num_tets, w.num_edges) == (r.num_nodes, r.num_tets, r.num_edges)
    assert (w.num_a, w.num_phi, w.num_ports, w.num_unknowns) == (r.num_a, r.num_phi, r.num_ports, r.n)
    rp, ci = r.pattern()
    np.testing.assert_array_equal(w.row_ptr, rp)
    np.testing.assert_array_equal(w.col_idx, ci)
    idx, co, fx = r.tet_dofs()
    np.testing.assert_array_equal(w.tet_idx, idx)
    np.testing.assert_array_equal(w.tet_coeff, co)
    np.testing.assert_array_equal(w.tet_fixed, fx)


@pytest.mark.parametrize("cells", [16, 24, 32])
def test_torus_matches_reference_pipeline(cells, ref_or_skip):
    """The torus with its internal current port: the cut's nodes read the
    port unknown from plus-side tets and a grounded zero from minus-side
    ones (src/dof_map.cpp:160-181), so the per-tet tables are where a wrong
    side would show."""
    w = ab.Workload.torus(cells)
    r = ref_or_skip.RefProblem.torus(cells, ordering=-1)
    assert (w.num_nodes, w.num_tets, w.num_edges) == (r.num_nodes, r.num_tets, r.num_edges)
    assert (w.num_a, w.num_phi, w.num_ports, w.num_unknowns) == (r.num_a, r.num_phi, r.num_ports, r.n)
    assert w.num_ports == 1 and list(w.port_current) == [1]
    rp, ci = r.pattern()
    np.testing.assert_array_equal(w.row_ptr, rp)
    np.testing.assert_array_equal(w.col_idx, ci)
    idx, co, fx = r.tet_dofs()
    np.testing.assert_array_equal(w.tet_idx, idx)
    np.testing.assert_array_equal(w.tet_coeff, co)
    np.testing.assert_array_equal(w.tet_fixed, fx)
    # both sides of the cut exist: some tets read the port unknown, and the
    # port unknown appears only through Phi entries
    port_row = int(w.port_row[0])
    assert (w.tet_idx.reshape(-1, 16)[:, 6:] == port_row).any()
    assert not (w.tet_idx.reshape(-1, 16)[:, :6] == port_row).any()


def test_torus_refusals():
    with pytest.raises(ab.AphiError, match="even number"):
        ab.Workload.torus(15)   # y = 0.5 is not a grid plane
    with pytest.raises(ab.AphiError, match="crosses no conductor"):
        ab.Workload.torus(12)   # the tube is too thin for a conductor face on the cut


def test_cylinder_6_sizes():
    """6^3 cells: the sizes the reference reports for this problem
    (1,296 tets, 1,358 unknowns = 1,081 A + 275 Phi + 2 ports, 15,164 stored)."""
    w = ab.Workload.cylinder(6)
    assert (w.num_tets, w.num_unknowns, w.num_a, w.num_phi, w.num_ports, w.nnz) == (
        1296, 1358, 1081, 275, 2, 15164)


def test_upper_pattern_well_formed():
    w = ab.Workload.cylinder(5)
    rp, ci = w.row_ptr, w.col_idx
    for r in range(w.num_unknowns):
        row = ci[rp[r]:rp[r + 1]]
        assert row.size > 0 and row[0] >= r
        assert np.all(np.diff(row) > 0)


def test_refuses_meshes_without_a_conductor():
    with pytest.raises(ab.AphiError):
        ab.Workload.cylinder(0)
    with pytest.raises(ab.AphiError):
        ab.Workload.cylinder(2)    # no centroid within r = 0.2: the reference refuses too


@pytest.mark.parametrize("kind,cells", [("cylinder", 12), ("torus", 16)])
def test_analysis_matches_reference_analyze(kind, cells, ref_or_skip):
    """The supernodal analysis recomputes the elimination tree and column
    counts from the pattern and the caller's permutation: on the reference's
    own analyze output (AMD, src/symbolic.cpp:126-194) both are equal, and the
    reference's tree and counts handed in are accepted."""
    r = getattr(ref_or_skip.RefProblem, kind)(cells)
    rp, ci = r.pattern()
    a = r.analysis()
    an = ab.Analysis(rp, ci, a["perm"], a["parent"], a["col_count"])
    parent, cc = an.etree()
    np.testing.assert_array_equal(parent, a["parent"])
    np.testing.assert_array_equal(cc, a["col_count"])
    assert int(an.info["nnz_l"]) == int(a["col_count"].astype(np.int64).sum())


def test_nested_dissection_is_a_fill_reducing_permutation():
    """Geometric nested dissection (an option beside the reference's AMD; the
    benchmark and the parity tests use AMD, which the reference's pipeline
    produces): a permutation of the unknowns, whose factor has less fill and
    far fewer flops than AMD's on the 16^3 cylinder."""
    w = ab.Workload.cylinder(16)
    nd = ab.nested_dissection(w.row_ptr, w.col_idx, w.dof_xyz)
    np.testing.assert_array_equal(np.sort(nd), np.arange(w.num_unknowns))
    a_nd = ab.Analysis(w.row_ptr, w.col_idx, nd).info
    a_amd = ab.Analysis(w.row_ptr, w.col_idx, ab.amd_ordering(w.row_ptr, w.col_idx)).info
    assert a_nd["nnz_l"] < 0.8 * a_amd["nnz_l"] and a_nd["flops"] < 0.5 * a_amd["flops"]


@pytest.mark.parametrize("kind,cells", [("cylinder", 4), ("cylinder", 8), ("cylinder", 12), ("torus", 16)])
def test_rcm_matches_reference(kind, cells, ref_or_skip):
    """The reverse Cuthill-McKee restatement gives the reference's own
    permutation (compute_ordering with Ordering::ReverseCuthillMcKee) bit for
    bit, voltage-port rows (isolated vertices) included."""
    w = getattr(ab.Workload, kind)(cells)
    r = getattr(ref_or_skip.RefProblem, kind)(cells, ordering=1)
    np.testing.assert_array_equal(ab.rcm_ordering(w.row_ptr, w.col_idx), r.analysis()["perm"])


@pytest.mark.parametrize("seed", range(6))
def test_rcm_and_amd_match_reference_on_random_patterns(seed, ref_or_skip):
    """Random upper patterns with several components, isolated unknowns and
    uneven degrees: both orderings equal the reference's."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(50, 600))
    rows = [{i} for i in range(n)]
    for i in range(n):
        for j in rng.integers(0, n, size=int(rng.integers(0, 5))):
            if j != i and rng.random() < 0.8:
                rows[min(i, j)].add(max(i, j))
    rp = np.zeros(n + 1, np.int32)
    ci = []
    for i, r in enumerate(rows):
        ci += sorted(r)
        rp[i + 1] = len(ci)
    ci = np.array(ci, np.int32)
    for code, fn in ((1, ab.rcm_ordering), (2, ab.amd_ordering)):
        ref = ref_or_skip.RefProblem.from_pattern(rp, ci, ordering=code)
        np.testing.assert_array_equal(fn(rp, ci), ref.analysis()["perm"])

"""The 24^3 and 32^3 reference fixtures (tests/golden/reference_*.npz,
written by the reference's own pipeline) against the host-side parts of this
repository, on the CPU: the workload generator and the AMD restatement must
give the reference's pattern and permutation bit for bit at the benchmarked
size, and the C oracle's refill the reference's refill. The GPU half of the
comparison (device refill and solutions) is tests/test_headline_parity_gpu.py."""
import numpy as np
import pytest

import aphi_b200 as ab
import oraclelib as orc
import reference_solutions as refsol


@pytest.mark.parametrize("mesh,cells", [("cylinder", 24), ("cylinder", 32), ("torus", 24), ("torus", 32)])
def test_pattern_permutation_and_oracle_refill_match_the_fixture(mesh, cells):
    fx = refsol.load(cells, mesh)
    assert fx is not None, f"{refsol.path(cells, mesh).name} is missing"
    w = ab.Workload.cylinder(cells) if mesh == "cylinder" else ab.Workload.torus(cells)
    assert w.row_ptr.size - 1 == fx["n"] and w.col_idx.size == fx["nnz"]
    assert refsol.sha(np.concatenate([w.row_ptr, w.col_idx]).astype(np.int32)) == fx["sha_pattern"]
    perm = ab.amd_ordering(w.row_ptr, w.col_idx)
    assert refsol.sha(perm) == fx["sha_perm"]
    k = 1
    v, b = orc.refill(ab.workload_arrays(w), fx["omegas"][k])
    assert refsol.sha(v) == fx["sha_values"][k] and refsol.sha(b) == fx["sha_rhs"][k]
    # the fixture's own solutions are solutions of those systems
    for j, rep in enumerate(fx["reports"]):
        # the torus's only source is its 1 A port: no FP64 solve reaches 1e-12 there
        assert rep["ok"] == 1 and rep["residual"] < (1e-12 if mesh == "cylinder" else 1e-3)
        assert np.isfinite(fx["x"][j]).all() and np.linalg.norm(fx["x"][j]) > 0

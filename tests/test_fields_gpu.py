"""Post-solve fields on the device against the reference's compute_fields
(src/postprocess.cpp:223-486) and potential_at_nodes (:42-126).

compute_fields is linear in the solution, so seeded random solution vectors
exercise every array: per tet A and E at the centroid, B = curl A, J = sigma E
and sigma; per P2 node Phi (the plus side on a cut), A, B, H, E, J with the
reference's side selection at material interfaces, the volume weights and the
interface flags. The device evaluates the reference's arithmetic in its order
and sums each node's contributions in the reference's tet order, so the
arrays are expected bit for bit; the test allows 1e-13 of each array's
largest entry and records how many match exactly."""
import numpy as np
import pytest
import torch

import aphi_b200 as ab

pytestmark = pytest.mark.gpu

COMPLEX = ["phi_node", "a_tet", "b_tet", "e_tet", "j_tet", "a_node", "b_node", "h_node", "e_node", "j_node"]


def compare(mine: dict, ref: dict):
    exact = 0
    for k in COMPLEX + ["sigma_tet", "vertex_weight"]:
        a = mine[k].cpu().numpy()
        b = ref[k]
        assert a.shape == b.shape, k
        scale = max(np.abs(b).max(initial=0.0), 1e-300)
        err = np.abs(a - b).max(initial=0.0)
        assert err <= 1e-13 * scale, (k, err, scale)
        exact += int(np.array_equal(a.view(np.float64) if np.iscomplexobj(a) else a,
                                    b.view(np.float64) if np.iscomplexobj(b) else b))
    np.testing.assert_array_equal(mine["on_interface"].cpu().numpy(), ref["on_interface"])
    return exact


def random_solution(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


@pytest.mark.parametrize("conditioning", [ab.COND_ROW_SCALED, ab.COND_SCALED_PHI])
def test_cylinder_fields_match_reference(conditioning, cuda, ref_or_skip):
    w = ab.Workload.cylinder(6)
    asm = ab.Assembly(ab.workload_arrays(w))
    fields = ab.Fields.of_workload(asm, w)
    r = ref_or_skip.RefProblem.cylinder(6, ordering=-1)
    omega = 2 * np.pi * 1e4
    x = random_solution(w.num_unknowns, 7)
    mine = fields.compute(torch.from_numpy(x).cuda(), omega, conditioning)
    ref = r.compute_fields(x, omega, conditioning)
    exact = compare(mine, ref)
    assert fields.num_interface_nodes == ref["num_interface_nodes"] > 0
    assert fields.num_orphans == ref["num_orphan_vertices"]
    assert exact >= 10, exact   # the arithmetic is the reference's: most arrays equal bit for bit


def test_torus_fields_match_reference(cuda, ref_or_skip):
    """The cut: Phi at a cut node is the plus side's value (the port's
    unknown), and each tet's E uses its own side's potential."""
    w = ab.Workload.torus(16)
    asm = ab.Assembly(ab.workload_arrays(w))
    fields = ab.Fields.of_workload(asm, w)
    r = ref_or_skip.RefProblem.torus(16, ordering=-1)
    omega = 2 * np.pi * 50.0
    x = random_solution(w.num_unknowns, 11)
    mine = fields.compute(torch.from_numpy(x).cuda(), omega, ab.COND_ROW_SCALED)
    ref = r.compute_fields(x, omega, ab.COND_ROW_SCALED)
    compare(mine, ref)
    port = x[int(w.port_row[0])]
    assert np.count_nonzero(ref["phi_node"] == port) > 0   # cut nodes report the port's unknown


def test_fields_refuse_a_wrong_solution(cuda):
    w = ab.Workload.cylinder(3)
    asm = ab.Assembly(ab.workload_arrays(w))
    fields = ab.Fields.of_workload(asm, w)
    with pytest.raises(ab.InvalidArgument):
        fields.compute(torch.zeros(w.num_unknowns - 1, dtype=torch.complex128, device="cuda"), 1.0)

"""Device assembly (element fill + fixed-order scatter) against the reference.

Element blocks: <= 1e-13 relative to kernel_AA/APhi/PhiPhi
(src/element_matrix.cpp:27-115) -- in fact bitwise, since the device kernels
round every operation as the host does. Assembled values and right-hand side:
bitwise equal to refill (src/assembly.cpp:468-494) on the same mesh."""
import numpy as np
import pytest

import aphi_b200 as ab

pytestmark = pytest.mark.gpu

OMEGAS = [2 * np.pi * 50.0, 2 * np.pi * 1.0e4, 2 * np.pi * 1.0e6]


def _rand_tets(rng, n):
    base = rng.uniform(-1, 1, size=(n, 1, 3))
    return base + rng.uniform(0, 1, size=(n, 4, 3))


def test_element_blocks_match_reference(cuda, ref_or_skip):
    rng = np.random.default_rng(1234)
    xyz = _rand_tets(rng, 64)
    xyz[0] = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]   # the unit tet of the reference's tests
    for sigma, eps_r, mu_r, omega in [(5.8e7, 1, 1, OMEGAS[0]), (0.0, 1, 1, OMEGAS[2]),
                                      (1.0, 4.0, 2.0, OMEGAS[1]), (5.8e7, 1, 1, 0.0)]:
        nu, alpha, beta = ab.element_coefficients(sigma, eps_r, mu_r, omega)
        aa, ap, pp = ab.element_blocks(xyz, nu, alpha, beta)
        for t in range(xyz.shape[0]):
            raa, rap, rpp = ref_or_skip.element_blocks(xyz[t], sigma, eps_r, mu_r, omega)
            for mine, theirs in ((aa[t], raa), (ap[t], rap), (pp[t], rpp)):
                scale = max(np.abs(theirs).max(), 1e-300)
                assert np.abs(mine - theirs).max() <= 1e-13 * scale
                np.testing.assert_array_equal(mine, theirs)  # bitwise


def test_unit_tet_curl_curl_known_answer(cuda):
    """Known answer of tests/test_element_matrix.cpp:101-134: on the unit tet
    the curl-curl block with nu = 1 is V * (c_i . c_j), the hand-computed dot
    products below over 6, to 1e-14; nu scales it linearly."""
    dots = np.array([[8, -4, -4, 4, 0, 4], [-4, 8, -4, -4, 4, 0], [-4, -4, 8, 0, -4, -4],
                     [4, -4, 0, 4, 0, 0], [0, 4, -4, 0, 4, 0], [4, 0, -4, 0, 0, 4]], float)
    xyz = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]], float)
    aa, ap, pp = ab.element_blocks(xyz, 1.0, 0j, 0j)
    assert np.abs(aa[0] - dots / 6.0).max() <= 1e-14
    assert abs(aa[0][0, 0] - 4.0 / 3.0) <= 1e-14
    assert not ap.any() and not pp.any()          # beta == 0 gives empty coupling blocks
    aa7, _, _ = ab.element_blocks(xyz, 7.0, 0j, 0j)
    assert abs(aa7[0][0, 0] - 7.0 * 4.0 / 3.0) <= 1e-13


@pytest.mark.parametrize("cells", [3, 6, 8])
@pytest.mark.parametrize("conditioning", [ab.COND_ROW_SCALED, ab.COND_SCALED_PHI])
def test_refill_bitwise_equal_to_reference(cells, conditioning, cuda, ref_or_skip):
    w = ab.Workload.cylinder(cells)
    asm = ab.Assembly(ab.workload_arrays(w))
    r = ref_or_skip.RefProblem.cylinder(cells, ordering=-1)
    for omega in OMEGAS:
        rv, rr = r.refill(omega, conditioning)
        v, b = asm.refill(omega, conditioning)
        v = v[0].cpu().numpy()
        b = b[0].cpu().numpy()
        np.testing.assert_array_equal(v.view(np.float64), rv.view(np.float64))
        np.testing.assert_array_equal(b.view(np.float64), rr.view(np.float64))


def test_refill_batch_equals_single(cuda):
    w = ab.Workload.cylinder(6)
    asm = ab.Assembly(ab.workload_arrays(w))
    om = np.geomspace(2 * np.pi * 50, 2 * np.pi * 1e6, 16)
    vb, bb = asm.refill(om)
    for k in (0, 7, 15):
        v1, b1 = asm.refill(om[k])
        assert bool((v1[0] == vb[k]).all()) and bool((b1[0] == bb[k]).all())


def test_refill_twice_is_identical(cuda):
    """refill clears before accumulating (src/assembly.cpp:262-266): a refill
    after another frequency equals a fresh one."""
    w = ab.Workload.cylinder(4)
    asm = ab.Assembly(ab.workload_arrays(w))
    v1, b1 = asm.refill(OMEGAS[0])
    asm.refill(OMEGAS[2], values=v1.clone(), rhs=b1.clone())
    v3, b3 = asm.refill(OMEGAS[0], values=v1, rhs=b1)
    v4, b4 = asm.refill(OMEGAS[0])
    assert bool((v3 == v4).all()) and bool((b3 == b4).all())


def test_refill_refusals(cuda):
    w = ab.Workload.cylinder(3)
    asm = ab.Assembly(ab.workload_arrays(w))
    with pytest.raises(ab.InvalidArgument):
        asm.refill(OMEGAS[0], ab.COND_NATURAL)          # unsymmetric into upper storage
    with pytest.raises(ab.InvalidArgument):
        asm.refill(0.0, ab.COND_ROW_SCALED)             # row scaling divides by j*omega


def test_refill_host_matches_device(cuda):
    w = ab.Workload.cylinder(4)
    asm = ab.Assembly(ab.workload_arrays(w))
    vh, bh = asm.refill_host(OMEGAS[1])
    v, b = asm.refill(OMEGAS[1])
    np.testing.assert_array_equal(vh, v[0].cpu().numpy())
    np.testing.assert_array_equal(bh, b[0].cpu().numpy())

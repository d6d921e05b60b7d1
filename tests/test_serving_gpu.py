"""The serving loop (aphi_b200.serving): continuous batching of requests of
different meshes, frequencies and excitation counts on one GPU.

Every request is answered to relative residual <= 1e-10, and its answer is
the same whether it was solved alone or in a mix with other requests: FP64
answers bit for bit (an entry's factorization and solve never read another
entry's data), mixed-precision answers to 1e-10 relative (the same FP32 +
COCG arithmetic per entry, converged to relative residual 1e-12)."""
import numpy as np
import pytest

import aphi_b200 as ab
from aphi_b200 import serving as sv

pytestmark = pytest.mark.gpu

CELLS = (4, 6, 8)


@pytest.fixture(scope="module")
def meshes(cuda):
    return {c: sv.MeshCache(c) for c in CELLS}


def trace(seed, count, f_hi=1e4):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        c = int(rng.choice(CELLS))
        f = float(np.exp(rng.uniform(np.log(50.0), np.log(f_hi))))
        k = int(rng.integers(1, 5))
        out.append(sv.Request(i, c, 2 * np.pi * f, np.exp(1j * rng.uniform(0, 2 * np.pi, size=k))))
    return out


def serve(meshes, requests, precision, workers):
    srv = sv.Server(meshes, precision, workers=workers, hbm_budget=20e9)
    for r in requests:
        r.arrival = srv.now()
        srv.submit(r)
    with srv.cv:
        while len(srv.finished) + len(srv.rejected) < len(requests):
            srv.cv.wait(timeout=0.1)
    srv.close()
    return srv


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mix_matches_alone(meshes, precision):
    reqs = trace(11, 24)
    srv = serve(meshes, reqs, precision, workers=2)
    assert not srv.rejected and all(not r.error for r in srv.finished)
    assert max(r.batch_size for r in reqs) > 1           # batching happened
    for r in reqs:
        assert r.x.shape == (len(r.voltages), meshes[r.cells].n)
        assert r.residual <= 1e-10, (r.rid, r.cells, r.omega, r.residual)
    for r in reqs[::3]:
        alone = sv.Request(r.rid, r.cells, r.omega, r.voltages.copy())
        serve(meshes, [alone], precision, workers=1)
        assert alone.batch_size == 1
        if precision == "fp64":
            np.testing.assert_array_equal(alone.x, r.x)
        else:
            err = np.linalg.norm(alone.x - r.x) / np.linalg.norm(r.x)
            assert err <= 1e-10, (r.rid, err)


def test_excitations_are_linear(meshes):
    """Two excitations V1, V2 of one request: x2 = (V2 / V1) x1."""
    r = sv.Request(0, 6, 2 * np.pi * 1e3, np.array([1.0 + 0j, np.exp(0.7j)]))
    serve(meshes, [r], "fp64", workers=1)
    np.testing.assert_allclose(r.x[1], np.exp(0.7j) * r.x[0], rtol=1e-12, atol=1e-12 * np.abs(r.x[0]).max())


def test_admission_refuses_what_it_cannot_hold(meshes):
    bad_mesh = sv.Request(0, 5, 2 * np.pi * 50.0, np.ones(1, complex))
    too_many = sv.Request(1, 4, 2 * np.pi * 50.0, np.ones(9, complex))
    ok = sv.Request(2, 4, 2 * np.pi * 50.0, np.ones(1, complex))
    srv = serve(meshes, [bad_mesh, too_many, ok], "fp64", workers=1)
    assert {r.rid for r in srv.rejected} == {0, 1}
    assert ok.residual <= 1e-10


def test_capacities_shrink_to_fit_the_budget(meshes):
    big = sv.Server(meshes, "mixed", workers=1, hbm_budget=50e9)
    tight = sv.Server(meshes, "mixed", workers=1, hbm_budget=0.02e9)
    assert big.footprint <= 50e9
    assert sum(tight.max_batch.values()) < sum(big.max_batch.values())
    big.close()
    tight.close()

"""Writes the golden fixtures in this folder from the reference itself.

    make -C oracle ref          # the reference compiled from its own sources
    python tests/golden/make_golden.py

Every number in the fixtures comes out of the reference's own code, called
through oracle/_ref/libaphi_ref.so (tests/refbridge.py): its mesh/DOF/sparsity
pipeline and AMD analysis, refill, compute_symmetric_equilibration,
factorize_ldlt, solve_symmetric and the three element kernels. The fixtures
pin the C oracle (tests/test_oracle.py) where the reference tree is absent.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import refbridge as rb  # noqa: E402

OMEGAS = 2 * np.pi * np.array([50.0, 1.0e3, 1.0e6])


def element_fixture():
    rng = np.random.default_rng(20261203)
    xyz = rng.uniform(-1, 1, size=(8, 1, 3)) + rng.uniform(0, 1, size=(8, 4, 3))
    xyz[0] = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]
    cases = np.array([[5.8e7, 1, 1, OMEGAS[0]], [0.0, 1, 1, OMEGAS[2]], [1.0, 4.0, 2.0, OMEGAS[1]],
                      [5.8e7, 1, 1, 0.0]])
    aa = np.zeros((len(cases), 8, 6, 6), np.complex128)
    ap = np.zeros((len(cases), 8, 6, 10), np.complex128)
    pp = np.zeros((len(cases), 8, 10, 10), np.complex128)
    for c, (sigma, eps_r, mu_r, omega) in enumerate(cases):
        for t in range(8):
            aa[c, t], ap[c, t], pp[c, t] = rb.element_blocks(xyz[t], sigma, eps_r, mu_r, omega)
    np.savez_compressed(HERE / "element_blocks.npz", xyz=xyz, cases=cases, aa=aa, ap=ap, pp=pp)


def cylinder_fixture(cells, omegas, with_factor):
    r = rb.RefProblem.cylinder(cells)
    rp, ci = r.pattern()
    an = r.analysis()
    out = dict(row_ptr=rp, col_idx=ci, perm=an["perm"], parent=an["parent"], col_count=an["col_count"],
               omegas=np.asarray(omegas), tet_idx=r.tet_dofs()[0])
    vals, rhs, xs, reps, ds = [], [], [], [], []
    for om in omegas:
        v, b = r.refill(om)
        x, rep = r.solve_symmetric(b)
        vals.append(v)
        rhs.append(b)
        xs.append(x)
        reps.append([rep[k] for k in ("ok", "backward_error", "residual", "equilibration_min",
                                      "equilibration_max", "smallest_pivot", "largest_pivot",
                                      "largest_multiplier", "factor_nnz", "columns_done")])
        ds.append(r.equilibration(10))
    out.update(values=np.array(vals), rhs=np.array(rhs), x=np.array(xs), report=np.array(reps), d=np.array(ds))
    if with_factor:
        r.set_values(vals[0])
        f = r.factorize()
        out.update(l_col_ptr=f["col_ptr"], l_row_index=f["row_index"], l_value=f["value"],
                   l_diagonal=f["diagonal"], l_stats=np.array([f["stats"][k] for k in (
                       "ok", "columns_done", "smallest_pivot", "largest_pivot", "largest_multiplier", "nnz")]))
    np.savez_compressed(HERE / f"cylinder{cells}.npz", **out)


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


def matrix_fixture():
    """Hand cases of tests/test_factorization.cpp (2x2, the zero pivot, a
    non-Hermitian complex symmetric 3x3) and seeded random patterns in the
    shape of its :169-213 (n 6..30, 12 % fill, diagonal shift 6n + 0.5n i)."""
    mats = [np.array([[2, 3], [3, 5]], np.complex128),
            np.array([[0, 1], [1, 0]], np.complex128),
            np.array([[4 + 1j, 1 - 2j, 0.5j], [1 - 2j, 3 - 1j, 2], [0.5j, 2, 5 + 3j]])]
    rng = np.random.default_rng(424242)
    for _ in range(6):
        n = int(rng.integers(6, 31))
        a = np.zeros((n, n), np.complex128)
        for i in range(n):
            for j in range(i + 1, n):
                if rng.random() < 0.12:
                    a[i, j] = a[j, i] = rng.normal() + 1j * rng.normal()
        a += np.diag(rng.normal(size=n) + 1j * rng.normal(size=n) + 6 * n + 0.5j * n)
        mats.append(a)
    out = {}
    for k, a in enumerate(mats):
        rp, ci, v = dense_to_upper(a)
        # the hand cases under the natural ordering, as the reference's tests
        # state them; the random ones under AMD
        r = rb.RefProblem.from_pattern(rp, ci, ordering=0 if k < 3 else 2)
        r.set_values(v)
        f = r.factorize()
        an = r.analysis()
        b = (np.arange(a.shape[0]) + 1.0) * (1 - 0.5j)
        x, rep = r.solve_symmetric(b, equil_iters=0) if f["stats"]["ok"] else (np.zeros(a.shape[0]), {})
        for key, val in dict(row_ptr=rp, col_idx=ci, values=v, perm=an["perm"], parent=an["parent"],
                             col_count=an["col_count"], l_col_ptr=f["col_ptr"], l_row_index=f["row_index"],
                             l_value=f["value"], l_diagonal=f["diagonal"], ok=np.array(f["stats"]["ok"]),
                             columns_done=np.array(f["stats"]["columns_done"]), b=b, x=x).items():
            out[f"m{k}_{key}"] = val
    out["count"] = np.array(len(mats))
    np.savez_compressed(HERE / "matrices.npz", **out)


if __name__ == "__main__":
    if not rb.available():
        sys.exit("oracle/_ref/libaphi_ref.so is missing: run `make -C oracle ref` where the reference tree is")
    element_fixture()
    cylinder_fixture(4, OMEGAS, with_factor=True)
    cylinder_fixture(6, OMEGAS[:1], with_factor=False)
    matrix_fixture()
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size, "bytes")

"""Writes the reference's own solutions of the benchmarked cylinder sweep
(and of the torus sweep of config 5).

    make -C oracle ref REF=<reference tree>
    python tests/golden/make_reference_solutions.py [--cells 24 32] [--jobs 6]
    python tests/golden/make_reference_solutions.py --mesh torus --cells 24 32

For each mesh (the Kuhn cylinder-in-box at 24^3 and 32^3 cells, reduced
A-Phi, row-scaled, AMD) and each chosen member of the 16-frequency sweep
(2*pi*geomspace(50 Hz, 1 MHz, 16)[k], k = 0, 8, 15: 50 Hz, 9.84 kHz, 1 MHz),
the reference's own pipeline runs through oracle/_ref/libaphi_ref.so
(tests/refbridge.py): mesh, gauge, DOF map, sparsity, AMD analysis, refill
(src/assembly.cpp:468-494) and solve_symmetric (src/factorization.cpp:332-398)
with 10 Ruiz iterations. One process per (mesh, frequency); a 32^3 solve takes
about 35 minutes of one core and 6.5 GB of host memory.

The torus (the copper torus with its 1 A internal cut port, reduced A-Phi,
row-scaled, AMD) uses members 0, 4 and 7 of its 8-point sweep (50 Hz .. 10
kHz). Each fixture `reference_<mesh><cells>.npz` holds:
  omegas, sweep_index          the frequencies (rad/s) and their sweep index
  x_shuffled                   the reference's solutions, complex128 [f, n],
                               stored byte-shuffled (all first bytes of every
                               double, then all second bytes, ...) so that
                               compression finds the exponent bytes' redundancy;
                               tests/reference_solutions.py undoes it
  report                       solve_symmetric's SolveReport per frequency
  sha_perm, sha_pattern        SHA-256 of the AMD permutation and of the CSR
                               pattern (row_ptr then col_idx, int32)
  sha_values, sha_rhs          SHA-256 of the refilled values and rhs per
                               frequency (complex128): the device refill must
                               reproduce these bytes
  n, nnz, nnz_l, factorize_ms  sizes, and the reference's factorization time
"""
import argparse
import hashlib
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

SWEEP_INDEX = (0, 8, 15)
# The torus (config 5): 8 log-spaced frequencies 50 Hz .. 10 kHz, members 0, 4, 7.
TORUS_INDEX = (0, 4, 7)
REPORT_KEYS = ("ok", "backward_error", "residual", "equilibration_min", "equilibration_max",
               "smallest_pivot", "largest_pivot", "largest_multiplier", "factor_nnz", "columns_done",
               "analyze_ms", "factorize_ms", "solve_ms")


def sweep_omegas(nfreq=16, f_lo=50.0, f_hi=1.0e6):
    return 2 * np.pi * np.geomspace(f_lo, f_hi, nfreq)


def torus_omegas():
    return sweep_omegas(8, 50.0, 1.0e4)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def shuffle_bytes(x: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(x, np.complex128).view(np.uint8).reshape(-1, 8)
    return np.ascontiguousarray(b.T)


def solve_one(task):
    mesh, cells, k = task
    import refbridge as rb
    t0 = time.time()
    r = rb.RefProblem.cylinder(cells) if mesh == "cylinder" else rb.RefProblem.torus(cells)
    rp, ci = r.pattern()
    an = r.analysis()
    om = float((sweep_omegas() if mesh == "cylinder" else torus_omegas())[k])
    v, b = r.refill(om)
    x, rep = r.solve_symmetric(b)
    print(f"{mesh} {cells} k {k}: {time.time() - t0:.0f} s, residual {rep['residual']:.2e}", flush=True)
    return dict(mesh=mesh, cells=cells, k=k, omega=om, x=x, report=[rep[key] for key in REPORT_KEYS],
                sha_perm=sha(an["perm"]), sha_pattern=sha(np.concatenate([rp, ci])),
                sha_values=sha(v), sha_rhs=sha(b), n=r.n, nnz=r.nnz, nnz_l=r.nnz_l)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, nargs="+", default=[24, 32])
    ap.add_argument("--mesh", default="cylinder", choices=["cylinder", "torus"])
    ap.add_argument("--jobs", type=int, default=6)
    args = ap.parse_args()
    import refbridge as rb
    if not rb.available():
        sys.exit("oracle/_ref/libaphi_ref.so is missing: run `make -C oracle ref REF=<reference tree>`")
    index = SWEEP_INDEX if args.mesh == "cylinder" else TORUS_INDEX
    tasks = [(args.mesh, c, k) for c in sorted(args.cells, reverse=True) for k in index]
    with mp.get_context("spawn").Pool(min(args.jobs, len(tasks))) as pool:
        results = pool.map(solve_one, tasks, chunksize=1)
    for cells in args.cells:
        rs = sorted([r for r in results if r["cells"] == cells], key=lambda r: r["k"])
        for key in ("sha_perm", "sha_pattern", "n", "nnz", "nnz_l"):
            assert len({r[key] for r in rs}) == 1, key
        x = np.array([r["x"] for r in rs])
        out = dict(omegas=np.array([r["omega"] for r in rs]), sweep_index=np.array([r["k"] for r in rs]),
                   x_shuffled=shuffle_bytes(x), x_shape=np.array(x.shape),
                   report=np.array([r["report"] for r in rs]), report_keys=np.array(REPORT_KEYS),
                   sha_perm=np.array(rs[0]["sha_perm"]), sha_pattern=np.array(rs[0]["sha_pattern"]),
                   sha_values=np.array([r["sha_values"] for r in rs]),
                   sha_rhs=np.array([r["sha_rhs"] for r in rs]),
                   n=np.array(rs[0]["n"]), nnz=np.array(rs[0]["nnz"]), nnz_l=np.array(rs[0]["nnz_l"]))
        path = HERE / f"reference_{args.mesh}{cells}.npz"
        np.savez_compressed(path, **out)
        print(path.name, path.stat().st_size, "bytes")


if __name__ == "__main__":
    main()

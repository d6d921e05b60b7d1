"""The reference's own solutions of the benchmarked cylinder sweep, as written
by tests/golden/make_reference_solutions.py (test infrastructure: the GPU
path is compared against these, never computed from them)."""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def path(cells: int, mesh: str = "cylinder") -> Path:
    return GOLDEN / f"reference_{mesh}{cells}.npz"


def load(cells: int, mesh: str = "cylinder") -> dict | None:
    """{omegas, sweep_index, x [f, n] complex128, reports [dict per f],
    sha_perm, sha_pattern, sha_values [f], sha_rhs [f], n, nnz, nnz_l}, or
    None when no fixture exists for this mesh."""
    p = path(cells, mesh)
    if not p.exists():
        return None
    z = np.load(p)
    shape = tuple(int(v) for v in z["x_shape"])
    x = np.ascontiguousarray(z["x_shuffled"].T).reshape(-1).view(np.complex128).reshape(shape)
    keys = [str(k) for k in z["report_keys"]]
    return dict(omegas=z["omegas"], sweep_index=z["sweep_index"], x=x,
                reports=[dict(zip(keys, row.tolist())) for row in z["report"]],
                sha_perm=str(z["sha_perm"]), sha_pattern=str(z["sha_pattern"]),
                sha_values=[str(s) for s in z["sha_values"]], sha_rhs=[str(s) for s in z["sha_rhs"]],
                n=int(z["n"]), nnz=int(z["nnz"]), nnz_l=int(z["nnz_l"]))

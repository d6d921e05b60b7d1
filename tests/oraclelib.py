"""ctypes view of oracle/liboracle.so, the C restatement of the reference's
hot path. Test infrastructure: used only as the checker."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "oracle" / "liboracle.so"
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, capture_output=True)
        _lib = C.CDLL(str(LIB))
        for name in ("or_coefficients", "or_element_blocks", "or_formulation_scales", "or_refill",
                     "or_equilibration", "or_factorize", "or_solve", "or_residuals", "or_solve_symmetric"):
            getattr(_lib, name).argtypes = None
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def _c128(a):
    return np.ascontiguousarray(a, np.complex128)


def coefficients(sigma, eps_r, mu_r, omega):
    out = np.zeros(5)
    lib().or_coefficients(C.c_double(sigma), C.c_double(eps_r), C.c_double(mu_r), C.c_double(omega), _p(out))
    return out[0], complex(out[1], out[2]), complex(out[3], out[4])


def element_blocks(xyz, nu, alpha, beta):
    x = np.ascontiguousarray(xyz, np.float64).reshape(12)
    a = np.array([alpha.real, alpha.imag])
    b = np.array([beta.real, beta.imag])
    aa = np.zeros(36, np.complex128)
    ap = np.zeros(60, np.complex128)
    pp = np.zeros(100, np.complex128)
    if lib().or_element_blocks(_p(x), C.c_double(nu), _p(a), _p(b), _p(aa), _p(ap), _p(pp)) != 0:
        raise ValueError("degenerate tet")
    return aa.reshape(6, 6), ap.reshape(6, 10), pp.reshape(10, 10)


def refill(arrays: dict, omega: float, conditioning: int = 1):
    """scatter_into over the workload's DOF tables (arrays as Workload.array names)."""
    A = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
    rp = _i32(A["row_ptr"])
    ci = _i32(A["col_idx"])
    n = rp.size - 1
    v = np.zeros(int(rp[-1]), np.complex128)
    r = np.zeros(n, np.complex128)
    rc = lib().or_refill(
        C.c_int(A["tets"].size // 4), _p(np.ascontiguousarray(A["xyz"], np.float64)), _p(_i32(A["tets"])),
        _p(_i32(A["tet_idx"])), _p(np.ascontiguousarray(A["tet_coeff"], np.float64)),
        _p(np.ascontiguousarray(A["tet_fixed"], np.float64)), C.c_int(A["material"].size // 3),
        _p(np.ascontiguousarray(A["material"], np.float64)), _p(_i32(A["body_ptr"])), _p(_i32(A["body_tets"])),
        C.c_int(A["port_row"].size), _p(_i32(A["port_current"])), _p(_i32(A["port_row"])),
        _p(np.ascontiguousarray(A["port_amplitude"], np.float64)),
        _p(np.ascontiguousarray(A["port_value"], np.float64)), C.c_int(n), _p(rp), _p(ci), C.c_double(omega),
        C.c_int(conditioning), _p(v), _p(r))
    if rc == -1:
        raise ValueError("refill: refused conditioning")
    if rc == -2:
        raise RuntimeError("refill: no slot for an entry")
    if rc == -3:
        raise ValueError("degenerate tet")
    return v, r


def equilibration(row_ptr, col_idx, values, iterations=10):
    rp, ci, v = _i32(row_ptr), _i32(col_idx), _c128(values)
    d = np.zeros(rp.size - 1)
    lib().or_equilibration(C.c_int(rp.size - 1), _p(rp), _p(ci), _p(v), C.c_int(iterations), _p(d))
    return d


def factorize(row_ptr, col_idx, values, perm, parent, col_count, pivot_floor=0.0):
    rp, ci, v = _i32(row_ptr), _i32(col_idx), _c128(values)
    pm, pa, cc = _i32(perm), _i32(parent), _i32(col_count)
    n = rp.size - 1
    nl = int(np.maximum(cc - 1, 0).sum())
    cp = np.zeros(n + 1, np.int32)
    ri = np.zeros(max(nl, 1), np.int32)
    lv = np.zeros(max(nl, 1), np.complex128)
    dg = np.zeros(n, np.complex128)
    stats = np.zeros(6)
    rc = lib().or_factorize(C.c_int(n), _p(rp), _p(ci), _p(v), _p(pm), _p(pa), _p(cc), C.c_double(pivot_floor),
                            _p(cp), _p(ri), _p(lv), _p(dg), _p(stats))
    if rc < 0:
        raise RuntimeError("factorize: a column received more entries than reserved")
    keys = ["ok", "columns_done", "smallest_pivot", "largest_pivot", "largest_multiplier", "nnz"]
    return dict(col_ptr=cp, row_index=ri[:nl], value=lv[:nl], diagonal=dg, stats=dict(zip(keys, stats.tolist())))


def solve(factor, perm, b):
    n = factor["diagonal"].size
    x = np.zeros(n, np.complex128)
    rc = lib().or_solve(C.c_int(n), _p(_i32(factor["col_ptr"])), _p(_i32(factor["row_index"])),
                        _p(_c128(factor["value"])), _p(_c128(factor["diagonal"])), _p(_i32(perm)), _p(_c128(b)),
                        _p(x))
    if rc != 0:
        raise RuntimeError("solve: zero pivot")
    return x


def residuals(row_ptr, col_idx, values, x, b):
    out = np.zeros(2)
    rp = _i32(row_ptr)
    lib().or_residuals(C.c_int(rp.size - 1), _p(rp), _p(_i32(col_idx)), _p(_c128(values)), _p(_c128(x)),
                       _p(_c128(b)), _p(out))
    return out[0], out[1]


REPORT = ["ok", "backward_error", "residual", "equilibration_min", "equilibration_max", "smallest_pivot",
          "largest_pivot", "largest_multiplier", "factor_nnz", "columns_done"]


def solve_symmetric(row_ptr, col_idx, values, b, perm, parent, col_count, equil_iters=10, pivot_floor=0.0):
    rp = _i32(row_ptr)
    n = rp.size - 1
    x = np.zeros(n, np.complex128)
    rep = np.zeros(10)
    rc = lib().or_solve_symmetric(C.c_int(n), _p(rp), _p(_i32(col_idx)), _p(_c128(values)), _p(_c128(b)),
                                  _p(_i32(perm)), _p(_i32(parent)), _p(_i32(col_count)), C.c_int(equil_iters),
                                  C.c_double(pivot_floor), _p(x), _p(rep))
    return rc == 0, x, dict(zip(REPORT, rep.tolist()))

"""ctypes view of oracle/_ref/libaphi_ref.so: the reference implementation,
compiled from its own sources by oracle/Makefile. Test infrastructure only --
it is the checker the GPU path is compared against."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
REF_LIB = ROOT / "oracle" / "_ref" / "libaphi_ref.so"

_ref = None


def available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_LIB))
        vp = C.c_void_p
        L.ref_kuhn_cylinder.restype = vp
        L.ref_kuhn_cylinder.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int]
        L.ref_kuhn_torus.restype = vp
        L.ref_kuhn_torus.argtypes = [C.c_int, C.c_double, C.c_int]
        L.ref_from_pattern.restype = vp
        L.ref_from_pattern.argtypes = [C.c_int, vp, vp, C.c_int]
        L.ref_free.argtypes = [vp]
        L.ref_last_error.restype = C.c_char_p
        for name in ("ref_sizes", "ref_nodes", "ref_tets", "ref_edges", "ref_dof_arrays",
                     "ref_tet_dofs", "ref_bodies", "ref_ports", "ref_pattern", "ref_analysis",
                     "ref_scatter_map"):
            getattr(L, name).argtypes = None
        L.ref_refill.argtypes = [vp, C.c_double, C.c_int, C.c_int, vp, vp, vp]
        L.ref_set_values.argtypes = [vp, vp]
        L.ref_solve_symmetric.argtypes = [vp, vp, C.c_int, C.c_double, vp, vp]
        L.ref_equilibration.argtypes = [vp, C.c_int, vp]
        L.ref_factorize.argtypes = [vp, C.c_double, vp, vp, vp, vp, vp]
        L.ref_element_blocks.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, vp, vp, vp]
        L.ref_body_tets.argtypes = [vp, C.c_int, vp]
        L.ref_compute_fields.argtypes = [vp, vp, C.c_double, C.c_int] + [vp] * 14
        _ref = L
    return _ref


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class RefProblem:
    """One problem held by the reference: the cylinder-in-box through its
    whole host pipeline, or a bare pattern analysed by it."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("reference: " + ref().ref_last_error().decode())
        self.h = C.c_void_p(handle)
        s = (C.c_longlong * 12)()
        ref().ref_sizes(self.h, s)
        (self.num_nodes, self.num_tets, self.num_edges, self.n, self.nnz, self.num_a,
         self.num_phi, self.num_ports, self.num_bodies, self.nnz_l, self.map_bytes,
         self.num_roots) = list(s)

    @classmethod
    def cylinder(cls, cells: int, v_top: float = 1.0, full_wave: bool = False, ordering: int = 2):
        return cls(ref().ref_kuhn_cylinder(cells, 1 if full_wave else 0, v_top, ordering))

    @classmethod
    def torus(cls, cells: int, current: float = 1.0, ordering: int = 2):
        return cls(ref().ref_kuhn_torus(cells, current, ordering))

    @classmethod
    def from_pattern(cls, row_ptr, col_idx, ordering: int = 2):
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        return cls(ref().ref_from_pattern(rp.size - 1, _p(rp), _p(ci), ordering))

    def __del__(self):
        try:
            ref().ref_free(self.h)
        except Exception:
            pass

    def pattern(self):
        rp = np.zeros(self.n + 1, np.int32)
        ci = np.zeros(self.nnz, np.int32)
        ref().ref_pattern(self.h, _p(rp), _p(ci))
        return rp, ci

    def analysis(self):
        a = [np.zeros(self.n, np.int32) for _ in range(4)]
        ref().ref_analysis(self.h, *map(_p, a))
        return dict(perm=a[0], iperm=a[1], parent=a[2], col_count=a[3])

    def compute_fields(self, x: np.ndarray, omega: float, conditioning: int = 1) -> dict:
        """The reference's compute_fields on solution x (complex128, n)."""
        x = np.ascontiguousarray(x, np.complex128)
        T, P = self.num_tets, self.num_nodes + self.num_edges
        out = {"phi_node": np.zeros(P, np.complex128), "sigma_tet": np.zeros(T),
               "vertex_weight": np.zeros(P), "on_interface": np.zeros(P, np.uint8)}
        for k in ("a_tet", "b_tet", "e_tet", "j_tet"):
            out[k] = np.zeros((T, 3), np.complex128)
        for k in ("a_node", "b_node", "h_node", "e_node", "j_node"):
            out[k] = np.zeros((P, 3), np.complex128)
        counts = np.zeros(2, np.int32)
        order = ["phi_node", "a_tet", "b_tet", "e_tet", "j_tet", "sigma_tet", "a_node", "b_node", "h_node",
                 "e_node", "j_node", "vertex_weight", "on_interface"]
        rc = ref().ref_compute_fields(self.h, _p(x), omega, conditioning, *[_p(out[k]) for k in order], _p(counts))
        if rc != 0:
            raise RuntimeError("reference: " + ref().ref_last_error().decode())
        out["num_interface_nodes"], out["num_orphan_vertices"] = int(counts[0]), int(counts[1])
        return out

    def tet_dofs(self):
        t = self.num_tets
        idx = np.zeros(16 * t, np.int32)
        co = np.zeros(16 * t)
        fx = np.zeros(20 * t)
        ref().ref_tet_dofs(self.h, _p(idx), _p(co), _p(fx))
        return idx, co, fx

    def refill(self, omega: float, conditioning: int = 1, use_map: bool = True):
        v = np.zeros(self.nnz, np.complex128)
        r = np.zeros(self.n, np.complex128)
        ms = np.zeros(1)
        rc = ref().ref_refill(self.h, omega, conditioning, 1 if use_map else 0, _p(v), _p(r), _p(ms))
        if rc != 0:
            raise ValueError(ref().ref_last_error().decode())
        self.refill_ms = float(ms[0])
        return v, r

    def set_values(self, values: np.ndarray):
        v = np.ascontiguousarray(values, np.complex128)
        ref().ref_set_values(self.h, _p(v))

    def solve_symmetric(self, rhs: np.ndarray, equil_iters: int = 10, pivot_floor: float = 0.0):
        b = np.ascontiguousarray(rhs, np.complex128)
        x = np.zeros(self.n, np.complex128)
        rep = np.zeros(16)
        rc = ref().ref_solve_symmetric(self.h, _p(b), equil_iters, pivot_floor, _p(x), _p(rep))
        if rc < 0:
            raise ValueError(ref().ref_last_error().decode())
        keys = ["ok", "backward_error", "residual", "equilibration_min", "equilibration_max",
                "smallest_pivot", "largest_pivot", "largest_multiplier", "factor_nnz",
                "columns_done", "analyze_ms", "factorize_ms", "solve_ms"]
        return x, dict(zip(keys, rep[:13].tolist()))

    def equilibration(self, iterations: int = 10):
        d = np.zeros(self.n)
        ref().ref_equilibration(self.h, iterations, _p(d))
        return d

    def factorize(self, pivot_floor: float = 0.0):
        n = self.n
        m = self.nnz_l - n
        cp = np.zeros(n + 1, np.int32)
        ri = np.zeros(max(m, 1), np.int32)
        lv = np.zeros(max(m, 1), np.complex128)
        dg = np.zeros(n, np.complex128)
        st = np.zeros(8)
        rc = ref().ref_factorize(self.h, pivot_floor, _p(cp), _p(ri), _p(lv), _p(dg), _p(st))
        if rc < 0:
            raise ValueError(ref().ref_last_error().decode())
        keys = ["ok", "columns_done", "smallest_pivot", "largest_pivot", "largest_multiplier",
                "nnz", "milliseconds"]
        return dict(col_ptr=cp, row_index=ri[:m], value=lv[:m], diagonal=dg,
                    stats=dict(zip(keys, st[:7].tolist())))


def element_blocks(xyz: np.ndarray, sigma: float, eps_r: float, mu_r: float, omega: float):
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(12)
    aa = np.zeros(36, np.complex128)
    ap = np.zeros(60, np.complex128)
    pp = np.zeros(100, np.complex128)
    rc = ref().ref_element_blocks(_p(xyz), sigma, eps_r, mu_r, omega, _p(aa), _p(ap), _p(pp))
    if rc != 0:
        raise ValueError(ref().ref_last_error().decode())
    return aa.reshape(6, 6), ap.reshape(6, 10), pp.reshape(10, 10)

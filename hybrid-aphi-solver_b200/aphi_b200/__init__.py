"""Python host layer over libaphi_b200.so (the C ABI in include/aphi_b200.h).

Mirrors the reference's hot-path interface (namespace aphi_solver,
include/aphi_solver/assembly.hpp and factorization.hpp): the same operations
under the same names, the same argument meaning and the same error behaviour
-- std::invalid_argument becomes InvalidArgument (a ValueError),
std::logic_error becomes LogicError, and a factorization that meets its pivot
floor returns False with stats.ok == False.

Device memory, streams and tensors come from PyTorch; all arithmetic runs in
the library's CUDA kernels. There is no CPU fallback: if the library or a GPU
is missing, every compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libaphi_b200.so"

OK = 0
ERR_BAD_SHAPE = 1
ERR_PATTERN_MISMATCH = 2
ERR_PIVOT_FLOOR = 3
ERR_NAN = 4
ERR_IR_STALL = 5
ERR_TIMEOUT = 6
ERR_OOM = 7
ERR_ADMISSION = 8
ERR_CUDA = 9
ERR_ZERO_PIVOT = 10
ERR_DEGENERATE_TET = 11
ERR_INVALID = 12

COND_NATURAL, COND_ROW_SCALED, COND_SCALED_PHI = 0, 1, 2
PREC_FP64, PREC_FP32 = 64, 32


class AphiError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class InvalidArgument(AphiError, ValueError):
    """std::invalid_argument in the reference."""


class LogicError(AphiError):
    """std::logic_error in the reference."""


class PivotFloor(AphiError):
    """The factorization stopped at a pivot at or below the floor."""


_lib = None


def lib() -> C.CDLL:
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run hybrid-aphi-solver_b200/build.py")
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


P = C.c_void_p
I = C.c_int
D = C.c_double
I64 = C.c_int64
PI = C.POINTER(C.c_int)
PD = C.POINTER(C.c_double)
PI64 = C.POINTER(C.c_int64)


class AssemblyDesc(C.Structure):
    _fields_ = [("num_nodes", I), ("num_tets", I), ("num_unknowns", I),
                ("xyz", PD), ("tets", PI), ("tet_idx", PI), ("tet_coeff", PD), ("tet_fixed", PD),
                ("num_bodies", I), ("material", PD), ("body_ptr", PI), ("body_tets", PI),
                ("num_ports", I), ("port_current", PI), ("port_row", PI),
                ("port_amplitude", PD), ("port_value", PD),
                ("upper_only", I), ("row_ptr", PI), ("col_idx", PI)]


class AnalysisOptions(C.Structure):
    _fields_ = [("relax_small", I), ("relax_fill", D), ("relax_max_width", I), ("small_front", I),
                ("group4_rows", I), ("group2_rows", I), ("tc_group4_rows", I), ("tc_group2_rows", I)]


class FactorStats(C.Structure):
    _fields_ = [("ok", I), ("columns_done", I), ("smallest_pivot", D), ("largest_pivot", D),
                ("largest_multiplier", D), ("nnz", I64), ("milliseconds", D),
                ("equilibration_min", D), ("equilibration_max", D)]


class IROptions(C.Structure):
    _fields_ = [("max_iters", I), ("tol", D), ("stall_ratio", D), ("krylov", I), ("rtol", D)]


class FieldsOut(C.Structure):
    _fields_ = [(name, P) for name in ("phi_node", "a_tet", "b_tet", "e_tet", "j_tet", "sigma_tet", "a_node",
                                       "b_node", "h_node", "e_node", "j_node", "vertex_weight", "on_interface")]


_SIGS = {
    "aphi_status_string": (C.c_char_p, [I]),
    "aphi_last_error": (C.c_char_p, []),
    "aphi_launch_count": (C.c_int64, []),
    "aphi_workload_cylinder": (I, [I, D, I, C.POINTER(P)]),
    "aphi_workload_torus": (I, [I, D, C.POINTER(P)]),
    "aphi_workload_free": (None, [P]),
    "aphi_workload_sizes": (I, [P, PI64]),
    "aphi_workload_array": (I, [P, C.c_char_p, C.POINTER(P), PI64]),
    "aphi_order_nested_dissection": (I, [I, PI, PI, PD, I, PI]),
    "aphi_order_amd": (I, [I, PI, PI, PI]),
    "aphi_order_rcm": (I, [I, PI, PI, PI]),
    "aphi_assembly_create": (I, [C.POINTER(AssemblyDesc), C.POINTER(P)]),
    "aphi_assembly_destroy": (I, [P]),
    "aphi_assembly_info": (I, [P, PI64]),
    "aphi_formulation_scales": (I, [I, D, PD, PI]),
    "aphi_refill": (I, [P, D, I, P, P, P]),
    "aphi_refill_batch": (I, [P, I, PD, I, P, P, P]),
    "aphi_refill_host": (I, [P, D, I, PD, PD]),
    "aphi_element_blocks": (I, [I, PD, D, PD, PD, PD, PD, PD]),
    "aphi_element_coefficients": (None, [D, D, D, D, PD]),
    "aphi_selftest_bounded_wait": (I, [C.c_longlong]),
    "aphi_fields_create": (I, [P, I, I, PI, C.POINTER(P)]),
    "aphi_fields_destroy": (I, [P]),
    "aphi_fields_sizes": (I, [P, PI64]),
    "aphi_fields_compute": (I, [P, D, I, P, C.POINTER(FieldsOut), P]),
    "aphi_analysis_default_options": (None, [C.POINTER(AnalysisOptions)]),
    "aphi_analysis_create": (I, [I, PI, PI, PI, PI, PI, C.POINTER(AnalysisOptions), C.POINTER(P)]),
    "aphi_analysis_destroy": (I, [P]),
    "aphi_analysis_info": (I, [P, PD]),
    "aphi_analysis_etree": (I, [P, PI, PI]),
    "aphi_factor_create": (I, [P, I, I, C.POINTER(P)]),
    "aphi_factor_destroy": (I, [P]),
    "aphi_factorize": (I, [P, P, I, D, C.POINTER(FactorStats), P]),
    "aphi_solve": (I, [P, I, P, P, P]),
    "aphi_factor_export": (I, [P, I, PI, PI, PD, PD, PD]),
    "aphi_residuals": (I, [P, I, I, P, P, P, PD, P]),
    "aphi_solve_refined": (I, [P, I, P, P, P, C.POINTER(IROptions), PI, PD, P]),
    "aphi_residuals_noalloc": (I, [P, I, I, P, P, P, PD, P]),
    "aphi_solve_symmetric_host": (I, [P, PD, PD, I, D, PD, PD]),
    "aphi_selftest_tc_tile": (I, [I, I, I, I, P, P, P]),
    "aphi_analysis_plan_stats": (I, [P, I, PI64, PI64, PD, PD]),
    "aphi_factor_profile": (I, [P, I]),
    "aphi_factor_set_batch": (I, [P, I]),
    "aphi_fronts_create": (I, [I, PI, PI, C.POINTER(AnalysisOptions), C.POINTER(P)]),
    "aphi_fronts_layout": (I, [P, PI64, PI64]),
    "aphi_factorize_fronts": (I, [P, P, C.POINTER(FactorStats), P]),
    "aphi_fronts_read": (I, [P, I, P, P, P]),
    "aphi_measure_peaks": (I, [PD]),
    "aphi_factorize_host": (I, [P, PD, I, D, C.POINTER(FactorStats)]),
    "aphi_solve_host": (I, [P, I, PD, PD]),
    "aphi_residuals_host": (I, [P, I, I, PD, PD, PD, PD]),
    "aphi_factor_profile_read": (I, [P, PD, PI64]),
    "aphi_assembly_create_device_setup": (I, [C.POINTER(AssemblyDesc), C.POINTER(P)]),
    "aphi_assembly_maps": (I, [P, PI64, PI, PI]),
    "aphi_pattern_build": (I, [I, I, PI, I, PI, I, PI, PI, C.c_int64, PI64]),
    "aphi_csc_solve_host": (I, [I, PI, PI, PD, PD, I, PD]),
    "aphi_csr_residuals_host": (I, [I, PI, PI, PD, I, PD, PD, PD]),
    "aphi_factor_set_tc_split": (I, [P, I]),
    "aphi_spmv": (I, [P, I, I, P, P, P, P]),
    "aphi_factor_profile_kinds": (I, [P, C.c_uint]),
    "aphi_selftest_tc_tile_split": (I, [I, I, I, I, I, P, P, P]),
}


def _declare(L: C.CDLL) -> None:
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args


def exported_symbols() -> list[str]:
    return list(_SIGS)


def launch_count() -> int:
    """Kernels the library has launched in this process."""
    return int(lib().aphi_launch_count())


def check(status: int) -> int:
    if status == OK:
        return status
    msg = lib().aphi_last_error().decode(errors="replace")
    if status == ERR_BAD_SHAPE:
        raise InvalidArgument(status, msg)
    if status in (ERR_PATTERN_MISMATCH, ERR_ZERO_PIVOT):
        raise LogicError(status, msg)
    if status == ERR_PIVOT_FLOOR:
        raise PivotFloor(status, msg)
    raise AphiError(status, f"{lib().aphi_status_string(status).decode()}: {msg}")


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def dptr(t) -> C.c_void_p:
    """Device pointer of a torch tensor (or None)."""
    return C.c_void_p(0 if t is None else t.data_ptr())


def stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    return C.c_void_p(stream.cuda_stream)


# ---------------------------------------------------------------- workloads
class Workload:
    """A synthetic problem's host-side inputs (numpy views): the cylinder-in-box
    or the torus with a cut port."""

    ARRAYS = {"xyz": np.float64, "tets": np.int32, "tet_idx": np.int32, "tet_coeff": np.float64,
              "tet_fixed": np.float64, "material": np.float64, "body_ptr": np.int32,
              "body_tets": np.int32, "port_current": np.int32, "port_row": np.int32,
              "port_amplitude": np.float64, "port_value": np.float64, "row_ptr": np.int32,
              "col_idx": np.int32, "edges": np.int32, "edge_index": np.int32,
              "phi_index": np.int32, "tet_edges": np.int32, "body_of_tet": np.int32,
              "dof_xyz": np.float64}

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        s = (C.c_int64 * 10)()
        check(lib().aphi_workload_sizes(self._h, s))
        (self.num_nodes, self.num_tets, self.num_edges, self.num_unknowns, self.nnz,
         self.num_a, self.num_phi, self.num_ports, self.num_bodies, _) = list(s)
        self._arrays = {}

    @classmethod
    def cylinder(cls, cells: int, v_top: float = 1.0, full_wave: bool = False) -> "Workload":
        h = P()
        check(lib().aphi_workload_cylinder(cells, v_top, 1 if full_wave else 0, C.byref(h)))
        return cls(h)

    @classmethod
    def torus(cls, cells: int, current: float = 1.0) -> "Workload":
        """The copper torus with one internal current port on its cut."""
        h = P()
        check(lib().aphi_workload_torus(cells, current, C.byref(h)))
        return cls(h)

    def array(self, name: str) -> np.ndarray:
        if name not in self._arrays:
            data = P()
            count = C.c_int64()
            check(lib().aphi_workload_array(self._h, name.encode(), C.byref(data), C.byref(count)))
            dt = np.dtype(self.ARRAYS[name])
            if count.value == 0:
                self._arrays[name] = np.zeros(0, dt)
            else:
                buf = (C.c_char * (count.value * dt.itemsize)).from_address(data.value)
                self._arrays[name] = np.frombuffer(buf, dtype=dt).copy()
        return self._arrays[name]

    def __getattr__(self, name):
        if name in Workload.ARRAYS:
            return self.array(name)
        raise AttributeError(name)

    def close(self):
        if self._h:
            lib().aphi_workload_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Fields:
    """Post-solve fields over an Assembly's mesh (compute_fields and
    potential_at_nodes' values, src/postprocess.cpp:42-126, 223-486): per tet
    A and E at the centroid, B = curl A, J = sigma E; per P2 node (vertices,
    then edge midpoints) Phi and volume-weighted A, B, H, E, J. The Assembly
    must stay alive as long as this object."""

    def __init__(self, assembly, num_nodes: int, num_edges: int, tet_edges):
        te = np.ascontiguousarray(tet_edges, np.int32)
        if te.size != 6 * assembly.num_tets:
            raise InvalidArgument(ERR_BAD_SHAPE, f"Fields: {te.size} tet edges for {assembly.num_tets} tets")
        self.assembly = assembly
        self._h = P()
        check(lib().aphi_fields_create(assembly._h, num_nodes, num_edges, _ptr(te, C.c_int), C.byref(self._h)))
        s = (C.c_int64 * 6)()
        check(lib().aphi_fields_sizes(self._h, s))
        self.num_tets, self.num_p2, self.num_vertices, self.num_edges, self.num_interface_nodes, \
            self.num_orphans = list(s)

    @classmethod
    def of_workload(cls, assembly, w: "Workload") -> "Fields":
        return cls(assembly, w.num_nodes, w.num_edges, w.tet_edges)

    def compute(self, x, omega: float, conditioning: int = COND_ROW_SCALED, stream=None) -> dict:
        """x: the solution, complex128 device tensor [N]. Returns device tensors."""
        import torch
        _expect_device(x, (self.assembly.num_unknowns,), "Fields.compute: x")
        T, Pn = self.num_tets, self.num_p2
        c = dict(dtype=torch.complex128, device="cuda")
        out = {"phi_node": torch.empty(Pn, **c), "sigma_tet": torch.empty(T, dtype=torch.float64, device="cuda"),
               "vertex_weight": torch.empty(Pn, dtype=torch.float64, device="cuda"),
               "on_interface": torch.empty(Pn, dtype=torch.uint8, device="cuda")}
        for k in ("a_tet", "b_tet", "e_tet", "j_tet"):
            out[k] = torch.empty((T, 3), **c)
        for k in ("a_node", "b_node", "h_node", "e_node", "j_node"):
            out[k] = torch.empty((Pn, 3), **c)
        fo = FieldsOut(**{k: dptr(v) for k, v in out.items()})
        check(lib().aphi_fields_compute(self._h, omega, conditioning, dptr(x), C.byref(fo), stream_ptr(stream)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().aphi_fields_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def assembly_desc_from(arrays: dict, upper_only: bool = True):
    """An AssemblyDesc over numpy arrays (kept alive by the returned tuple)."""
    keep = {}

    def arr(name, dt):
        a = np.ascontiguousarray(arrays[name], dtype=dt)
        keep[name] = a
        return a

    xyz = arr("xyz", np.float64)
    tets = arr("tets", np.int32)
    tet_idx = arr("tet_idx", np.int32)
    tet_coeff = arr("tet_coeff", np.float64)
    tet_fixed = arr("tet_fixed", np.float64)
    material = arr("material", np.float64)
    body_ptr = arr("body_ptr", np.int32)
    body_tets = arr("body_tets", np.int32)
    port_current = arr("port_current", np.int32)
    port_row = arr("port_row", np.int32)
    port_amplitude = arr("port_amplitude", np.float64)
    port_value = arr("port_value", np.float64)
    row_ptr = arr("row_ptr", np.int32)
    col_idx = arr("col_idx", np.int32)
    d = AssemblyDesc()
    d.num_nodes = xyz.size // 3
    d.num_tets = tets.size // 4
    d.num_unknowns = row_ptr.size - 1
    d.xyz, d.tets, d.tet_idx = _ptr(xyz, C.c_double), _ptr(tets, C.c_int), _ptr(tet_idx, C.c_int)
    d.tet_coeff, d.tet_fixed = _ptr(tet_coeff, C.c_double), _ptr(tet_fixed, C.c_double)
    d.num_bodies = material.size // 3
    d.material, d.body_ptr, d.body_tets = (_ptr(material, C.c_double), _ptr(body_ptr, C.c_int),
                                           _ptr(body_tets, C.c_int))
    d.num_ports = port_row.size
    d.port_current, d.port_row = _ptr(port_current, C.c_int), _ptr(port_row, C.c_int)
    d.port_amplitude, d.port_value = _ptr(port_amplitude, C.c_double), _ptr(port_value, C.c_double)
    d.upper_only = 1 if upper_only else 0
    d.row_ptr, d.col_idx = _ptr(row_ptr, C.c_int), _ptr(col_idx, C.c_int)
    return d, keep


def pattern_build(n: int, tet_idx, diag_rows=(), upper_only: bool = True):
    """build_sparsity (src/sparsity.cpp:19-136) on the device from the tets' 16
    DOF indices each plus the voltage-port diagonal rows: (row_ptr, col_idx)."""
    ti = np.ascontiguousarray(tet_idx, np.int32)
    dr = np.ascontiguousarray(diag_rows, np.int32)
    rp = np.zeros(n + 1, np.int32)
    nnz = C.c_int64(0)
    cap = max(16 * ti.size, 1)
    ci = np.zeros(cap, np.int32)
    rc = lib().aphi_pattern_build(n, ti.size // 16, ti.ctypes.data_as(PI), dr.size, dr.ctypes.data_as(PI),
                                  1 if upper_only else 0, rp.ctypes.data_as(PI), ci.ctypes.data_as(PI), cap,
                                  C.byref(nnz))
    if rc == ERR_BAD_SHAPE and nnz.value > cap:
        ci = np.zeros(nnz.value, np.int32)
        rc = lib().aphi_pattern_build(n, ti.size // 16, ti.ctypes.data_as(PI), dr.size, dr.ctypes.data_as(PI),
                                      1 if upper_only else 0, rp.ctypes.data_as(PI), ci.ctypes.data_as(PI),
                                      nnz.value, C.byref(nnz))
    check(rc)
    return rp, ci[: nnz.value]


def workload_arrays(w: Workload) -> dict:
    return {k: w.array(k) for k in Workload.ARRAYS}


def nested_dissection(row_ptr, col_idx, xyz, leaf: int = 64) -> np.ndarray:
    """Fill-reducing permutation (new -> old) by geometric nested dissection."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    xy = np.ascontiguousarray(xyz, np.float64)
    perm = np.zeros(rp.size - 1, np.int32)
    check(lib().aphi_order_nested_dissection(rp.size - 1, _ptr(rp, C.c_int), _ptr(ci, C.c_int),
                                             _ptr(xy, C.c_double), leaf, _ptr(perm, C.c_int)))
    return perm


def amd_ordering(row_ptr, col_idx) -> np.ndarray:
    """The reference's AMD permutation (new -> old), compute_ordering with
    Ordering::ApproximateMinimumDegree (src/ordering.cpp:539-556)."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    perm = np.zeros(rp.size - 1, np.int32)
    check(lib().aphi_order_amd(rp.size - 1, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(perm, C.c_int)))
    return perm


def rcm_ordering(row_ptr, col_idx) -> np.ndarray:
    """The reference's reverse Cuthill-McKee permutation (new -> old),
    compute_ordering with Ordering::ReverseCuthillMcKee
    (src/ordering.cpp:105-218, :512-537), bit for bit."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    perm = np.zeros(rp.size - 1, np.int32)
    check(lib().aphi_order_rcm(rp.size - 1, _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(perm, C.c_int)))
    return perm


# ---------------------------------------------------------------- assembly
def formulation_scales(conditioning: int, omega: float):
    """formulation_scales (src/assembly.cpp:12-45): (row, column, symmetric)."""
    rc = (C.c_double * 4)()
    sym = C.c_int()
    check(lib().aphi_formulation_scales(conditioning, omega, rc, C.byref(sym)))
    return complex(rc[0], rc[1]), complex(rc[2], rc[3]), bool(sym.value)


def element_coefficients(sigma: float, eps_r: float, mu_r: float, omega: float):
    out = (C.c_double * 5)()
    lib().aphi_element_coefficients(sigma, eps_r, mu_r, omega, out)
    return out[0], complex(out[1], out[2]), complex(out[3], out[4])


def element_blocks(xyz: np.ndarray, nu: float, alpha: complex, beta: complex):
    """kernel_AA / kernel_APhi / kernel_PhiPhi on the device for tets xyz[T,4,3]."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 12)
    t = xyz.shape[0]
    aa = np.zeros((t, 36), np.complex128)
    ap = np.zeros((t, 60), np.complex128)
    pp = np.zeros((t, 100), np.complex128)
    a = (C.c_double * 2)(alpha.real, alpha.imag)
    b = (C.c_double * 2)(beta.real, beta.imag)
    check(lib().aphi_element_blocks(t, _ptr(xyz, C.c_double), nu, a, b,
                                    aa.view(np.float64).ctypes.data_as(PD),
                                    ap.view(np.float64).ctypes.data_as(PD),
                                    pp.view(np.float64).ctypes.data_as(PD)))
    return aa.reshape(t, 6, 6), ap.reshape(t, 6, 10), pp.reshape(t, 10, 10)


class Assembly:
    """Device assembly for one mesh: refill at any frequency (refill,
    src/assembly.cpp:453-494). Values and rhs are complex128 device tensors."""

    def __init__(self, arrays: dict, upper_only: bool = True, device_setup: bool = True):
        """device_setup: build the per-mesh scatter maps (term destinations
        and slot -> term lists) on the device; False builds the same arrays on
        the host."""
        desc, keep = assembly_desc_from(arrays, upper_only)
        self.num_tets = int(desc.num_tets)
        self._h = P()
        create = lib().aphi_assembly_create_device_setup if device_setup else lib().aphi_assembly_create
        check(create(C.byref(desc), C.byref(self._h)))
        info = (C.c_int64 * 4)()
        check(lib().aphi_assembly_info(self._h, info))
        self.nnz, self.num_unknowns, self.num_terms, self.device_bytes = list(info)

    def refill(self, omega, conditioning=COND_ROW_SCALED, values=None, rhs=None, stream=None):
        import torch
        omegas = np.atleast_1d(np.asarray(omega, dtype=np.float64))
        nf = omegas.size
        if values is None:
            values = torch.empty((nf, self.nnz), dtype=torch.complex128, device="cuda")
        if rhs is None:
            rhs = torch.empty((nf, self.num_unknowns), dtype=torch.complex128, device="cuda")
        check(lib().aphi_refill_batch(self._h, nf, _ptr(omegas, C.c_double), conditioning,
                                      dptr(values), dptr(rhs), stream_ptr(stream)))
        return values, rhs

    def maps(self):
        """(term_off [T+1], dest_ptr [nnz+N+1], dest_terms [num_terms]) on the host."""
        to = np.zeros(self.num_tets + 1, np.int64)
        dp = np.zeros(self.nnz + self.num_unknowns + 1, np.int32)
        dt = np.zeros(max(self.num_terms, 1), np.int32)
        check(lib().aphi_assembly_maps(self._h, to.ctypes.data_as(PI64), dp.ctypes.data_as(PI),
                                       dt.ctypes.data_as(PI)))
        return to, dp, dt[: self.num_terms]

    def refill_host(self, omega: float, conditioning=COND_ROW_SCALED):
        v = np.zeros(self.nnz, np.complex128)
        r = np.zeros(self.num_unknowns, np.complex128)
        check(lib().aphi_refill_host(self._h, omega, conditioning, v.view(np.float64).ctypes.data_as(PD),
                                     r.view(np.float64).ctypes.data_as(PD)))
        return v, r

    def close(self):
        if getattr(self, "_h", None):
            lib().aphi_assembly_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- analysis
def default_analysis_options() -> AnalysisOptions:
    o = AnalysisOptions()
    lib().aphi_analysis_default_options(C.byref(o))
    return o


class Analysis:
    """Supernodal schedule for one pattern + permutation (the reference's
    SolverAnalysis, include/aphi_solver/symbolic.hpp:69-92, consumed as input).

    perm is the reference's Permutation::perm (new -> old); parent and
    col_count, when given, must equal this pattern's elimination tree and
    column counts under perm (LogicError otherwise)."""

    INFO = ["n", "nnz_upper", "nnz_l", "stored", "supernodes", "levels", "max_rows", "max_width",
            "flops", "cb_pool", "factor_bytes_fp64", "num_roots"]

    def __init__(self, row_ptr, col_idx, perm=None, parent=None, col_count=None, options=None):
        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        n = rp.size - 1
        pm = None if perm is None else np.ascontiguousarray(perm, np.int32)
        pa = None if parent is None else np.ascontiguousarray(parent, np.int32)
        cc = None if col_count is None else np.ascontiguousarray(col_count, np.int32)
        opt = options if options is not None else default_analysis_options()
        self._keep = (rp, ci)
        self._h = P()
        nul = C.POINTER(C.c_int)()
        check(lib().aphi_analysis_create(
            n, _ptr(rp, C.c_int), _ptr(ci, C.c_int),
            nul if pm is None else _ptr(pm, C.c_int), nul if pa is None else _ptr(pa, C.c_int),
            nul if cc is None else _ptr(cc, C.c_int), C.byref(opt), C.byref(self._h)))
        info = (C.c_double * 12)()
        check(lib().aphi_analysis_info(self._h, info))
        self.info = dict(zip(self.INFO, list(info)))
        self.n = n
        self.nnz = int(self.info["nnz_upper"])
        self.row_ptr, self.col_idx = rp, ci

    PLAN_KINDS = ["extend_add", "small_front", "diag_block", "panel_rows", "update_wide", "fwd_gather", "fwd_diag",
                  "fwd_update", "bwd_update", "bwd_diag", "update_panel", "update_tc", "tc_split",
                  "dmma_scale"]

    def plan_stats(self, plan: int, flops: bool = False) -> dict:
        """{kind: (launches, items)} of launch plan `plan` (0 factorization,
        1 tensor-core factorization, 2 forward solve, 3 backward solve); with
        flops=True, {kind: (launches, items, useful_flops, executed_flops)}
        (flops counted for the update kinds only)."""
        nk = len(self.PLAN_KINDS)
        la = np.zeros(nk, np.int64)
        it = np.zeros(nk, np.int64)
        us = np.zeros(nk)
        ex = np.zeros(nk)
        check(lib().aphi_analysis_plan_stats(self._h, plan, la.ctypes.data_as(PI64), it.ctypes.data_as(PI64),
                                             us.ctypes.data_as(PD) if flops else None,
                                             ex.ctypes.data_as(PD) if flops else None))
        if flops:
            return {k: (int(a), int(b), float(u), float(e)) for k, a, b, u, e in zip(self.PLAN_KINDS, la, it, us, ex)
                    if a}
        return {k: (int(a), int(b)) for k, a, b in zip(self.PLAN_KINDS, la, it) if a}

    def etree(self):
        parent = np.zeros(self.n, np.int32)
        cc = np.zeros(self.n, np.int32)
        check(lib().aphi_analysis_etree(self._h, _ptr(parent, C.c_int), _ptr(cc, C.c_int)))
        return parent, cc

    def close(self):
        if getattr(self, "_h", None):
            lib().aphi_analysis_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # Python-side mirror of factorize_ldlt / solve / solve_symmetric lives in
    # the Factor class and the module functions below.


STATS_KEYS = ["ok", "columns_done", "smallest_pivot", "largest_pivot", "largest_multiplier", "nnz",
              "milliseconds", "equilibration_min", "equilibration_max"]


class Fronts:
    """Independent dense fronts (the supernode-update microbenchmark's
    shape): front s has rows[s] rows, the first widths[s] its pivots. A
    Factor made from it factorizes the fronts' panels and leaves each
    contribution block as -L21 D L21^T (see aphi_fronts_create)."""

    def __init__(self, rows, widths, options=None):
        self.rows = np.ascontiguousarray(rows, np.int32)
        self.widths = np.ascontiguousarray(widths, np.int32)
        opt = options if options is not None else default_analysis_options()
        self._h = P()
        check(lib().aphi_fronts_create(self.rows.size, _ptr(self.rows, C.c_int), _ptr(self.widths, C.c_int),
                                       C.byref(opt), C.byref(self._h)))
        info = (C.c_double * 12)()
        check(lib().aphi_analysis_info(self._h, info))
        self.info = dict(zip(Analysis.INFO, list(info)))
        self.n = int(self.info["n"])
        self.stored, self.cb_pool = int(self.info["stored"]), int(self.info["cb_pool"])
        self.panel_offset = np.zeros(self.rows.size, np.int64)
        self.cb_offset = np.zeros(self.rows.size, np.int64)
        check(lib().aphi_fronts_layout(self._h, self.panel_offset.ctypes.data_as(PI64),
                                       self.cb_offset.ctypes.data_as(PI64)))

    PLAN_KINDS = Analysis.PLAN_KINDS

    def plan_stats(self, plan: int, flops: bool = False) -> dict:
        return Analysis.plan_stats(self, plan, flops)

    def close(self):
        if getattr(self, "_h", None):
            lib().aphi_analysis_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stats_dict(s: FactorStats) -> dict:
    return {k: getattr(s, k) for k in STATS_KEYS}


def _expect_device(t, shape, what: str, contiguous: bool = True) -> None:
    """The device entry points take raw pointers, so a tensor of the wrong
    shape, type or placement would be read past its end: refuse it here."""
    import torch
    ok = (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.complex128
          and tuple(t.shape) == tuple(shape) and (t.is_contiguous() or not contiguous))
    if not ok:
        got = (f"{tuple(t.shape)} {t.dtype} on {t.device}" if isinstance(t, torch.Tensor) else type(t).__name__)
        raise InvalidArgument(ERR_BAD_SHAPE, f"{what}: expected a {'contiguous ' if contiguous else ''}complex128 "
                                             f"CUDA tensor of shape {tuple(shape)}, got {got}")


class Factor:
    """`batch` numeric factorizations sharing one Analysis, resident on the
    device (factorize_ldlt, src/factorization.cpp:109-218, run as a
    supernodal multifrontal LDL^T with no pivoting and no conjugation)."""

    def __init__(self, analysis: Analysis, precision: int = PREC_FP64, batch: int = 1):
        self.analysis = analysis
        self.precision = precision
        self.batch = batch
        self.capacity = batch
        self.n = analysis.n
        self._h = P()
        check(lib().aphi_factor_create(analysis._h, precision, batch, C.byref(self._h)))
        self.stats = []

    def factorize(self, values, equilibration_iterations: int = 10, pivot_floor: float = 0.0,
                  stream=None) -> bool:
        """values: complex128 device tensor [batch, nnz]. Returns False (with
        self.stats[k]['ok'] == 0) if any entry met the pivot floor."""
        _expect_device(values, (self.batch, self.analysis.nnz), "factorize: values")
        st = (FactorStats * self.batch)()
        rc = lib().aphi_factorize(self._h, dptr(values), equilibration_iterations, pivot_floor, st,
                                  stream_ptr(stream))
        self.stats = [_stats_dict(s) for s in st]
        if rc == ERR_PIVOT_FLOOR:
            return False
        check(rc)
        return True

    def solve(self, b, x=None, stream=None):
        """b: complex128 device tensor [batch, nrhs, n] (or [batch, n])."""
        import torch
        squeeze = b.dim() == 2
        bb = b.unsqueeze(1) if squeeze else b
        nrhs = bb.shape[1]
        _expect_device(bb, (self.batch, nrhs, self.n), "solve: b", contiguous=False)
        bb = bb.contiguous()
        if x is None:
            x = torch.empty_like(bb)
        else:
            _expect_device(x.unsqueeze(1) if x.dim() == 2 else x, (self.batch, nrhs, self.n), "solve: x")
        check(lib().aphi_solve(self._h, nrhs, dptr(bb), dptr(x), stream_ptr(stream)))
        return x.squeeze(1) if squeeze else x

    def solve_refined(self, values, b, tol=1e-16, max_iters=40, stall_ratio=0.5, krylov=True, rtol=1e-14,
                      stream=None):
        """Refined solve (aphi_solve_refined): preconditioned COCG (krylov=True)
        or plain refinement, in FP64 on the original systems. Returns x, the
        iterations and backward error per system, and whether all converged."""
        import torch
        squeeze = b.dim() == 2
        bb = (b.unsqueeze(1) if squeeze else b).contiguous()
        nrhs = bb.shape[1]
        _expect_device(values, (self.batch, self.analysis.nnz), "solve_refined: values")
        _expect_device(bb, (self.batch, nrhs, self.n), "solve_refined: b")
        x = torch.empty_like(bb)
        it = (C.c_int * (self.batch * nrhs))()
        be = (C.c_double * (self.batch * nrhs))()
        opt = IROptions(max_iters, tol, stall_ratio, 1 if krylov else 0, rtol)
        rc = lib().aphi_solve_refined(self._h, nrhs, dptr(values), dptr(bb), dptr(x), C.byref(opt), it, be,
                                      stream_ptr(stream))
        if rc not in (OK, ERR_IR_STALL):
            check(rc)
        x = x.squeeze(1) if squeeze else x
        return x, np.array(list(it)).reshape(self.batch, nrhs), np.array(list(be)).reshape(self.batch, nrhs), rc == OK

    def factorize_fronts(self, panels, stream=None) -> bool:
        """Dense fronts: panels is a complex128 device tensor [batch, stored]
        in the Fronts' panel layout. Returns False if a pivot was zero."""
        st = (FactorStats * self.batch)()
        rc = lib().aphi_factorize_fronts(self._h, dptr(panels), st, stream_ptr(stream))
        self.stats = [_stats_dict(s) for s in st]
        if rc == ERR_PIVOT_FLOOR:
            return False
        check(rc)
        return True

    def read_fronts(self, k: int = 0, stream=None):
        """Entry k's factored panels and contribution blocks (complex128 device tensors)."""
        import torch
        a = self.analysis
        panels = torch.empty(a.stored, dtype=torch.complex128, device="cuda")
        cb = torch.empty(max(a.cb_pool, 1), dtype=torch.complex128, device="cuda")
        check(lib().aphi_fronts_read(self._h, k, dptr(panels), dptr(cb), stream_ptr(stream)))
        return panels, cb

    def set_tc_split(self, split: int) -> None:
        """FP32 factors: TF32 pieces per operand in the tensor-core update (3 or 2)."""
        check(lib().aphi_factor_set_tc_split(self._h, split))
        self.tc_split = split

    def set_batch(self, batch: int) -> None:
        """Process `batch` (1..capacity) entries from now on, without reallocating."""
        check(lib().aphi_factor_set_batch(self._h, batch))
        self.batch = batch

    def profile(self, enable: bool = True, kinds=None) -> None:
        """Per-kind device timing of later factorizations and solves (clears
        the totals); kinds: names of the kinds to time (all when None)."""
        if enable and kinds:
            mask = 0
            for k in kinds:
                mask |= 1 << Analysis.PLAN_KINDS.index(k)
            check(lib().aphi_factor_profile_kinds(self._h, mask))
        else:
            check(lib().aphi_factor_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        """{kind: (launches, ms)} accumulated since profile(True)."""
        ms = np.zeros(len(Analysis.PLAN_KINDS))
        la = np.zeros(len(Analysis.PLAN_KINDS), np.int64)
        check(lib().aphi_factor_profile_read(self._h, ms.ctypes.data_as(PD), la.ctypes.data_as(PI64)))
        return {k: (int(a), float(t)) for k, a, t in zip(Analysis.PLAN_KINDS, la, ms) if a}

    def export(self, k: int = 0) -> dict:
        """Entry k in the reference's SymmetricFactor layout (strictly lower
        CSC, rows ascending, caller's permuted numbering) plus D and the
        equilibration vector."""
        n = self.n
        nl = int(self.analysis.info["nnz_l"]) - n
        cp = np.zeros(n + 1, np.int32)
        ri = np.zeros(max(nl, 1), np.int32)
        val = np.zeros(max(nl, 1), np.complex128)
        dg = np.zeros(n, np.complex128)
        ds = np.zeros(n)
        check(lib().aphi_factor_export(self._h, k, _ptr(cp, C.c_int), _ptr(ri, C.c_int),
                                       val.view(np.float64).ctypes.data_as(PD),
                                       dg.view(np.float64).ctypes.data_as(PD), _ptr(ds, C.c_double)))
        return dict(col_ptr=cp, row_index=ri[:nl], value=val[:nl], diagonal=dg, d=ds)

    def close(self):
        if getattr(self, "_h", None):
            lib().aphi_factor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def residuals(analysis: Analysis, values, x, b, stream=None) -> np.ndarray:
    """[batch, nrhs, 2]: relative_residual and backward_error per solution
    (src/factorization.cpp:315-329, :401-416), on the original system."""
    bb = b.unsqueeze(1) if b.dim() == 2 else b
    xx = x.unsqueeze(1) if x.dim() == 2 else x
    batch, nrhs = bb.shape[0], bb.shape[1]
    _expect_device(values, (batch, analysis.nnz), "residuals: values")
    _expect_device(bb, (batch, nrhs, analysis.n), "residuals: b", contiguous=False)
    _expect_device(xx, (batch, nrhs, analysis.n), "residuals: x", contiguous=False)
    out = np.zeros((batch, nrhs, 2))
    check(lib().aphi_residuals(analysis._h, batch, nrhs, dptr(values), dptr(xx.contiguous()),
                               dptr(bb.contiguous()), out.ctypes.data_as(PD), stream_ptr(stream)))
    return out


def spmv(analysis: Analysis, values, x, stream=None):
    """A x on the original upper-stored systems (device tensors; x [batch, n]
    or [batch, nrhs, n]), SparseSymmetric::matvec
    (include/aphi_solver/sparse_symmetric.hpp:120-136)."""
    import torch
    xx = (x.unsqueeze(1) if x.dim() == 2 else x).contiguous()
    batch, nrhs = xx.shape[0], xx.shape[1]
    _expect_device(values, (batch, analysis.nnz), "spmv: values")
    _expect_device(xx, (batch, nrhs, analysis.n), "spmv: x")
    y = torch.empty_like(xx)
    check(lib().aphi_spmv(analysis._h, batch, nrhs, dptr(values), dptr(xx), dptr(y), stream_ptr(stream)))
    return y.squeeze(1) if x.dim() == 2 else y


def measure_peaks() -> dict:
    """Arithmetic peaks of the current device in TFLOP/s (aphi_measure_peaks)."""
    out = np.zeros(5)
    check(lib().aphi_measure_peaks(out.ctypes.data_as(PD)))
    return dict(zip(["fp64_dmma", "fp64_dfma", "fp32_ffma", "tf32_tc_n64", "tf32_tc_n256"], out.tolist()))


def bounded_wait_selftest(spin_limit: int = 1 << 12) -> int:
    """Status of aphi_selftest_bounded_wait: a device wait that nothing ends,
    bounded like the tensor-core tile's. ERR_TIMEOUT is the expected answer."""
    return int(lib().aphi_selftest_bounded_wait(spin_limit))


def tc_tile_selftest(P: np.ndarray, i0: int, j0: int, d: np.ndarray | None = None, split: int = 3) -> np.ndarray:
    """One tensor-core update tile: the 128 x 64 complex64 block
    sum_k (P[i0 + r, k] d[k]) P[j0 + c, k] (rows of P past its end read as
    zero), computed by the kernel the FP32 factorization uses, with its
    operands split into `split` TF32 pieces."""
    Pc = np.asfortranarray(P, np.complex64)
    rows, K = Pc.shape
    dd = None if d is None else np.ascontiguousarray(d, np.complex64)
    out = np.zeros((64, 128), np.complex64)
    check(lib().aphi_selftest_tc_tile_split(split, rows, K, i0, j0, C.c_void_p(Pc.ctypes.data),
                                            None if dd is None else C.c_void_p(dd.ctypes.data),
                                            C.c_void_p(out.ctypes.data)))
    return out.T


REPORT_KEYS = ["ok", "backward_error", "residual", "equilibration_min", "equilibration_max", "smallest_pivot",
               "largest_pivot", "largest_multiplier", "factor_nnz", "columns_done", "analyze_ms", "factorize_ms",
               "solve_ms"]


def solve_symmetric(analysis: Analysis, values: np.ndarray, b: np.ndarray, equilibration_iterations: int = 10,
                    pivot_floor: float = 0.0):
    """solve_symmetric (src/factorization.cpp:332-398) on host arrays:
    returns (ok, x, report). ok is False, with the report filled as far as it
    got, when the factorization met its pivot floor."""
    v = np.ascontiguousarray(values, np.complex128)
    bb = np.ascontiguousarray(b, np.complex128)
    if bb.size != analysis.n:
        raise InvalidArgument(ERR_BAD_SHAPE, f"solve_symmetric: the right-hand side has {bb.size} entries "
                                             f"for a matrix of {analysis.n} rows")
    x = np.zeros(analysis.n, np.complex128)
    rep = np.zeros(13)
    rc = lib().aphi_solve_symmetric_host(analysis._h, v.view(np.float64).ctypes.data_as(PD),
                                         bb.view(np.float64).ctypes.data_as(PD), equilibration_iterations,
                                         pivot_floor, x.view(np.float64).ctypes.data_as(PD),
                                         rep.ctypes.data_as(PD))
    report = dict(zip(REPORT_KEYS, rep.tolist()))
    if rc == ERR_PIVOT_FLOOR:
        return False, x, report
    check(rc)
    return True, x, report


# ---------------------------------------------------------------- frequency sweeps
class SweepSolver:
    """Frequency batching over one mesh: every frequency of a sweep shares the
    pattern and the supernodal schedule, so fills, factorizations and refined
    solves run as batched launches over all of them.

    precision="mixed": the frequencies are factorized together in FP32 and
    refined by FP64 preconditioned COCG on the original systems to the FP64
    direct solve's own residual level (rtol); an entry whose refinement
    stalls (cond(A) * eps(FP32) too large -- the high-frequency end of the
    cylinder sweep) is refactorized in FP64 automatically. The solver
    remembers the lowest frequency at which that happened: later sweeps send
    that frequency and every higher one straight to FP64 instead of spending
    an FP32 factorization on them (predict=False disables this).
    precision="fp64": the plain FP64 factorization for every entry (the
    drop-in path).

    Factor batches are sized to the entries they hold, split evenly into at
    most fp64_batch (FP64) or fp32_batch (FP32) entries per factorization, so
    no factorization is spent on padding.

    tc_split: TF32 pieces per FP32 operand in the tensor-core updates of the
    FP32 factors. 2 (hh + hl + lh, half the tensor-core work of 3) by default:
    on the 32^3 sweep it needs the same refinement iterations as 3 (4-13).

    overlap=True: entries predicted to need FP64 are factorized and solved on
    a side stream, from a second host thread, while the FP32 entries are
    being factorized and refined (results are the same either way; only the
    schedule changes).

    fp64_refine=True refines every FP64-factorized entry (fallbacks included)
    by COCG preconditioned with its own FP64 factor, to the same rtol / tol:
    for systems whose plain FP64 direct solve stops short of the residual
    target (the torus with its cut port: ~4e-10 at 50 Hz).
    """

    def __init__(self, analysis: Analysis, assembly: Assembly, batch: int, precision: str = "mixed",
                 fp64_batch: int = 8, rtol: float = 1e-14, tol: float = 1e-16, max_iters: int = 40,
                 fp32_batch: int | None = None, predict: bool = True, fp64_refine: bool = False,
                 tc_split: int = 2, overlap: bool = True):
        if precision not in ("mixed", "fp64"):
            raise InvalidArgument(ERR_BAD_SHAPE, f"SweepSolver: precision {precision!r} is not 'mixed' or 'fp64'")
        self.analysis, self.assembly = analysis, assembly
        self.batch, self.precision = batch, precision
        self.rtol, self.tol, self.max_iters = rtol, tol, max_iters
        self.fp64_batch = max(1, min(fp64_batch, batch))
        self.fp32_batch = max(1, min(fp32_batch or batch, batch))
        self.predict = predict
        self.fp64_refine = fp64_refine
        self.tc_split = tc_split
        self.overlap = overlap
        self._side_stream = None
        self.stall_omega = None      # lowest frequency whose FP32 refinement stalled
        self._factors = {}
        self._profile = False
        self._profile_kinds = None
        self._prof_done = {}         # precision -> {kind: (launches, ms)} of factors since replaced
        self.factorized = {PREC_FP32: 0, PREC_FP64: 0}   # entries factorized since profile(True)

    def _factor(self, precision: int, size: int) -> Factor:
        """The resident factor of this precision holding `size` entries: kept
        across calls and chunks, reallocated only when it must grow."""
        f = self._factors.get(precision)
        if f is None or f.capacity < size:
            if f is not None:
                self._fold_profile(precision, f)
                f.close()
                self._factors.pop(precision)
            f = Factor(self.analysis, precision, size)
            if precision == PREC_FP32:
                f.set_tc_split(self.tc_split)
            if self._profile:
                f.profile(True, self._profile_kinds)
            self._factors[precision] = f
        if f.batch != size:
            f.set_batch(size)
        return f

    def _fold_profile(self, precision, f):
        if not self._profile:
            return
        acc = self._prof_done.setdefault(precision, {})
        for k, (n, ms) in f.profile_read().items():
            a = acc.get(k, (0, 0.0))
            acc[k] = (a[0] + n, a[1] + ms)

    def profile(self, enable: bool = True, kinds=None) -> None:
        """Per-kind device timing of every factorization from now on (only the
        named kinds when `kinds` is given)."""
        self._profile = enable
        self._profile_kinds = kinds
        self._prof_done = {}
        self.factorized = {PREC_FP32: 0, PREC_FP64: 0}
        for f in self._factors.values():
            f.profile(enable, kinds)

    def profile_read(self) -> dict:
        """{"fp32" | "fp64": {kind: (launches, ms)}} since profile(True)."""
        out = {}
        for prec, name in ((PREC_FP32, "fp32"), (PREC_FP64, "fp64")):
            acc = dict(self._prof_done.get(prec, {}))
            f = self._factors.get(prec)
            if f is not None:
                for k, (n, ms) in f.profile_read().items():
                    a = acc.get(k, (0, 0.0))
                    acc[k] = (a[0] + n, a[1] + ms)
            if acc:
                out[name] = acc
        return out

    @property
    def f32(self):
        return self._factors.get(PREC_FP32)

    @property
    def f64(self):
        return self._factors.get(PREC_FP64)

    @staticmethod
    def _chunks(idx, cap):
        nb = -(-len(idx) // cap) if idx else 0
        size = -(-len(idx) // nb) if nb else 0
        return [idx[c:c + size] for c in range(0, len(idx), size)] if size else []

    def _fp64_chunk(self, idx, vals, rhs, stream):
        import torch
        f = self._factor(PREC_FP64, len(idx))
        sel = torch.tensor(idx, device=vals.device)
        v = vals.index_select(0, sel)
        f.factorize(v, 10, 0.0, stream=stream)
        self.factorized[PREC_FP64] += len(idx)
        iters = [0] * len(idx)
        if self.fp64_refine:
            xs, it, _, _ = f.solve_refined(v, rhs.index_select(0, sel), tol=self.tol, rtol=self.rtol,
                                           max_iters=self.max_iters, stream=stream)
            iters = [int(it[q, 0]) for q in range(len(idx))]
        else:
            xs = f.solve(rhs.index_select(0, sel), stream=stream)
        return xs, iters

    def _start_fp64(self, todo, vals, rhs, stream):
        """FP64 factorizations and solves of `todo` on the side stream, in a
        thread; returns (thread, box) with box["parts"] = [(idx, x, iters)] and
        box["event"] recorded on the side stream after the last of them."""
        import threading
        import torch
        if self._side_stream is None:
            self._side_stream = torch.cuda.Stream(device=vals.device)
        side = self._side_stream
        ready = torch.cuda.Event()
        ready.record(stream or torch.cuda.current_stream())
        box = {"parts": [], "error": None, "event": torch.cuda.Event()}

        def run():
            try:
                with torch.cuda.stream(side):
                    side.wait_event(ready)
                    for idx in self._chunks(sorted(todo), self.fp64_batch):
                        xs, iters = self._fp64_chunk(idx, vals, rhs, side)
                        box["parts"].append((idx, xs, iters))
                    box["event"].record(side)
            except Exception as e:  # re-raised by the caller after join
                box["error"] = e

        t = threading.Thread(target=run, daemon=True)
        t.start()
        return t, box

    def close(self):
        for f in self._factors.values():
            f.close()
        self._factors = {}

    def solve(self, omegas, conditioning=COND_ROW_SCALED, stream=None, values=None, rhs=None):
        """Returns (x [batch, n], values, rhs, per-entry reports), all device
        tensors. values/rhs, when given, are already-assembled systems (the
        drop-in flow, where refill handed them to the host and back);
        otherwise the sweep is assembled on the device first."""
        import torch
        om = np.asarray(omegas, dtype=np.float64)
        if om.size != self.batch:
            raise InvalidArgument(ERR_BAD_SHAPE, f"SweepSolver: {om.size} frequencies for a batch of {self.batch}")
        if values is None or rhs is None:
            vals, rhs = self.assembly.refill(om, conditioning, stream=stream)
        else:
            vals = values
        reports = [dict(omega=float(w), precision="fp64", iterations=0, predicted_fp64=False) for w in om]
        x = torch.empty_like(rhs)
        fp32_idx, todo = [], []
        for k in range(self.batch):
            if self.precision == "mixed" and not (self.predict and self.stall_omega is not None
                                                  and om[k] >= self.stall_omega):
                fp32_idx.append(k)
            else:
                todo.append(k)
                reports[k]["predicted_fp64"] = self.precision == "mixed"
        # Entries known in advance to need FP64 are factorized on a side stream
        # from a second host thread while the FP32 entries are factorized and
        # refined: the FP32 factorization's small in-panel and split launches
        # and the refinement's latency-bound solves leave much of the device to
        # the FP64 factorization. Each precision has its own contribution-block
        # workspace in the analysis, so the two factorizations run at the same
        # time; the solves do not touch the workspaces.
        side = None
        if self.overlap and todo and fp32_idx:
            side = self._start_fp64(todo, vals, rhs, stream)
            todo = []
        for idx in self._chunks(fp32_idx, self.fp32_batch):
            f = self._factor(PREC_FP32, len(idx))
            whole = len(idx) == self.batch
            sel = None if whole else torch.tensor(idx, device=vals.device)
            v = vals if whole else vals.index_select(0, sel)
            b = rhs if whole else rhs.index_select(0, sel)
            f.factorize(v, 10, 0.0, stream=stream)
            self.factorized[PREC_FP32] += len(idx)
            xs, iters, berr, _ = f.solve_refined(v, b, tol=self.tol, rtol=self.rtol, max_iters=self.max_iters,
                                                 stream=stream)
            res = residuals(self.analysis, v, xs, b, stream=stream)
            if whole:
                x.copy_(xs)
            else:
                x.index_copy_(0, sel, xs)
            for q, k in enumerate(idx):
                reports[k]["iterations"] = int(iters[q, 0])
                if res[q, 0, 0] <= self.rtol and res[q, 0, 1] <= self.tol:
                    reports[k]["precision"] = "fp32"
                else:
                    todo.append(k)
                    if self.stall_omega is None or om[k] < self.stall_omega:
                        self.stall_omega = float(om[k])
        if side is not None:
            thread, box = side
            thread.join()
            if box.get("error") is not None:
                raise box["error"]
            done_ev, parts = box["event"], box["parts"]
            main = stream or torch.cuda.current_stream()
            main.wait_event(done_ev)
            for idx, xs, iters in parts:
                xs.record_stream(main)   # read here, allocated on the side stream
                x.index_copy_(0, torch.tensor(idx, device=vals.device), xs)
                for q, k in enumerate(idx):
                    reports[k]["iterations"] = iters[q]
        todo.sort()
        for idx in self._chunks(todo, self.fp64_batch):
            f = self._factor(PREC_FP64, len(idx))
            sel = torch.tensor(idx, device=vals.device)
            v = vals.index_select(0, sel)
            f.factorize(v, 10, 0.0, stream=stream)
            self.factorized[PREC_FP64] += len(idx)
            if self.fp64_refine:
                xs, iters, _, _ = f.solve_refined(v, rhs.index_select(0, sel), tol=self.tol, rtol=self.rtol,
                                                  max_iters=self.max_iters, stream=stream)
                for q, k in enumerate(idx):
                    reports[k]["iterations"] = int(iters[q, 0])
            else:
                xs = f.solve(rhs.index_select(0, sel), stream=stream)
            x.index_copy_(0, sel, xs)
        return x, vals, rhs, reports

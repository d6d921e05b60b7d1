"""Per-mesh setup on the device against the host builders.

build_sparsity (src/sparsity.cpp:19-136) run on the device from the tets' DOF
tables must give the workload's pattern bit for bit (the host generator's
pattern equals the reference pipeline's: tests/test_workload.py), upper and
full storage; the scatter maps built on the device (term destinations and
slot -> term lists, src/assembly.cpp:196-232) must equal the host-built
maps, and refill through them must give the same bits; a pattern missing an
entry the scatter needs is refused with the entry named."""
import ctypes as C

import numpy as np
import pytest

import aphi_b200 as ab

pytestmark = pytest.mark.gpu

MESHES = [("cylinder", 3), ("cylinder", 6), ("cylinder", 12), ("torus", 16)]


def workload(kind, cells):
    return ab.Workload.cylinder(cells) if kind == "cylinder" else ab.Workload.torus(cells)


def voltage_rows(arrays):
    cur = np.asarray(arrays["port_current"])
    return np.asarray(arrays["port_row"])[cur == 0]


@pytest.mark.parametrize("kind,cells", MESHES)
def test_device_pattern_equals_host(kind, cells, cuda):
    w = workload(kind, cells)
    a = ab.workload_arrays(w)
    rp, ci = ab.pattern_build(w.row_ptr.size - 1, a["tet_idx"], voltage_rows(a))
    np.testing.assert_array_equal(rp, w.row_ptr)
    np.testing.assert_array_equal(ci, w.col_idx)
    # full storage: the upper pattern and its mirror
    n = rp.size - 1
    rpf, cif = ab.pattern_build(n, a["tet_idx"], voltage_rows(a), upper_only=False)
    rows = np.repeat(np.arange(n), np.diff(w.row_ptr))
    pairs = np.unique(np.concatenate([rows * n + w.col_idx, w.col_idx * n + rows]).astype(np.int64))
    np.testing.assert_array_equal(np.diff(rpf), np.bincount(pairs // n, minlength=n))
    np.testing.assert_array_equal(cif, (pairs % n).astype(np.int32))


@pytest.mark.parametrize("kind,cells", MESHES)
def test_device_scatter_maps_equal_host(kind, cells, cuda):
    w = workload(kind, cells)
    a = ab.workload_arrays(w)
    host = ab.Assembly(a, device_setup=False)
    dev = ab.Assembly(a, device_setup=True)
    assert (host.num_terms, host.nnz, host.num_unknowns) == (dev.num_terms, dev.nnz, dev.num_unknowns)
    for x, y in zip(host.maps(), dev.maps()):
        np.testing.assert_array_equal(x, y)
    om = 2 * np.pi * np.array([50.0, 3.0e4, 1.0e6])
    vh, bh = host.refill(om)
    vd, bd = dev.refill(om)
    assert bool((vh == vd).all()) and bool((bh == bd).all())


def test_missing_slot_is_refused_with_the_entry(cuda):
    """The cylinder's pattern with one off-diagonal entry taken out: the
    device map builder must refuse it (PATTERN_MISMATCH) and name the entry,
    as the host builder does, rather than drop the term."""
    w = ab.Workload.cylinder(3)
    a = dict(ab.workload_arrays(w))
    rp, ci = np.array(a["row_ptr"]), np.array(a["col_idx"])
    r = 5
    k = rp[r] + 1                         # an entry right of the diagonal
    c = int(ci[k])
    a["col_idx"] = np.delete(ci, k)
    a["row_ptr"] = np.concatenate([rp[: r + 1], rp[r + 1:] - 1]).astype(np.int32)
    desc, keep = ab.assembly_desc_from(a)
    h = C.c_void_p()
    rc = ab.lib().aphi_assembly_create_device_setup(C.byref(desc), C.byref(h))
    assert rc == ab.ERR_PATTERN_MISMATCH
    msg = ab.lib().aphi_last_error().decode()
    assert f"no slot for entry ({r}, {c})" in msg

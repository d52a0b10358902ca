"""The C-ABI library loads and exports every entry point declared in include/slopegpu.h.
No compute call is made here (CPU-only machine)."""
import ctypes
import os
import re

from slope_stability_octave_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(sg_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_all_declared_symbols():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_every_declared_symbol():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_abi_version_and_error_string():
    L = _lib.lib()
    assert L.sg_abi_version() >= 1
    assert isinstance(L.sg_last_error(), bytes)


def test_argument_errors_need_no_device():
    """Invalid arguments are rejected before any device work."""
    L = _lib.lib()
    rc = L.sg_reduction_dev(None, None, None, 1.0, b"Z", 10, None, None, None)
    assert rc == -1 and b"Davis" in L.sg_last_error()
    rc = L.sg_constitutive3d(None, None, None, None, None, None, ctypes.c_int64(-1), None, None, None)
    assert rc == -1


def test_new_entry_points_reject_bad_arguments_without_device():
    """The fused residual and the AMG clone check their arguments before any device work."""
    L = _lib.lib()
    rc = L.sg_residual_dev(None, None, None, None, None, None, None, None, None)
    assert rc == -1 and b"null" in L.sg_last_error()
    out = ctypes.c_void_p()
    rc = L.sg_amg_clone(None, ctypes.byref(out))
    assert rc == -1 and out.value is None
    rc = L.sg_amg_update(None, None, None)
    assert rc == -1


def test_noalloc_capacity_matches_header():
    """The allocation-free entry point's capacity is the header's SG_NOALLOC_MAX_POINTS; its
    GPU test uses the same figure."""
    text = open(os.path.join(ROOT, "include", "slopegpu.h")).read()
    m = re.search(r"#define\s+SG_NOALLOC_MAX_POINTS\s+(\d+)", text)
    assert m
    import tests.test_zz_no_alloc as t
    assert t.MAX_POINTS == int(m.group(1))
    L = _lib.lib()
    rc = L.sg_constitutive3d_noalloc(None, None, None, None, None, None, ctypes.c_int64(int(m.group(1)) + 1),
                                     None, None, None)
    assert rc == -1 and m.group(1).encode() in L.sg_last_error()


def test_ijv_instances_reject_bad_arguments_without_device():
    """The id-keyed preconditioner entry points check ids and sizes before any device work."""
    L = _lib.lib()
    buf = (ctypes.c_int64 * 8)()
    assert L.sg_amg_ijv_info(b"no_such_id", buf, 8) == -4
    assert L.sg_amg_update_values(b"no_such_id", None, 0, None) == -4
    assert L.sg_amg_apply_host(b"no_such_id", buf, buf, 1) == -4
    rc = L.sg_amg_setup_ijv(b"x", None, None, None, 0, 0, None, 0, None, 3, None, 0, 0, None)
    assert rc == -1 and b"n must be positive" in L.sg_last_error()
    rc = L.sg_amg_setup_ijv(b"x", buf, buf, buf, 1, 4, None, 0, None, 4, None, 0, 0, None)
    assert rc == -1 and b"num_functions" in L.sg_last_error()
    rc = L.sg_amg_setup_ijv(b"", buf, buf, buf, 1, 4, None, 0, None, 3, None, 0, 0, None)
    assert rc == -1
    assert L.sg_amg_clear(b"no_such_id") == 0
    assert L.sg_amg_ijv_info(None, buf, 8) == 0 and buf[0] == 0


def test_seepage_entry_points_reject_bad_arguments_without_device():
    """The seepage entry points check their arguments before any device work."""
    L = _lib.lib()
    rc = L.sg_seepage_system_dev(None, None, None, None, None, None, 9.81, 2, None, None, None, None)
    assert rc == -1 and b"null" in L.sg_last_error()
    rc = L.sg_point_gradient_dev(None, None, None, None)
    assert rc == -1
    rc = L.sg_seepage_saturation_dev(None, None, None, None, None, None, None)
    assert rc == -1
    out = ctypes.c_void_p()
    rc = L.sg_mesh_bsr_scalar(None, ctypes.byref(out))
    assert rc == -1 and out.value is None

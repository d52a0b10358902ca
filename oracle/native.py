"""ctypes bindings for the oracle's C restatement and the compiled reference MEX files.

Test infrastructure only (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")

_lib = None


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and, when the reference tree is present, _ref/*.so)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref_root = os.environ.get("SG_REF_ROOT", "/root/reference/slope_stability")
    if ref and os.path.isdir(ref_root):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={ref_root}"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        vp = C.c_void_p
        L.orc_constitutive3d.argtypes = [vp] * 6 + [C.c_int64, vp, vp, vp]
        L.orc_constitutive2d.argtypes = [vp] * 6 + [C.c_int64, vp, vp, vp]
        L.orc_reduction.argtypes = [vp, vp, vp, C.c_double, C.c_char, C.c_int64, vp, vp]
        L.orc_assemble.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int64, C.c_int, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


def constitutive(dim, E, c_bar, sin_phi, shear, bulk, lame, want_ds=True):
    """Oracle S, DS, branch for a point batch.  E is (n_strain, n) column-major, i.e.
    numpy shape (n, n_strain) row-major: pass E with shape (n, 6) or (n, 3)."""
    E = _c(E)
    n = E.shape[0]
    ns_out, nds = (6, 36) if dim == 3 else (4, 9)
    S = np.zeros((n, ns_out))
    DS = np.zeros((n, nds)) if want_ds else None
    br = np.zeros(n, np.uint8)
    args = [_p(E)] + [_p(_c(x)) for x in (c_bar, sin_phi, shear, bulk, lame)]
    fn = lib().orc_constitutive3d if dim == 3 else lib().orc_constitutive2d
    fn(*args, n, _p(S), _p(DS), _p(br))
    return S, DS, br


def reduction(c0, phi, psi, lam, davis="B"):
    c0, phi, psi = _c(c0), _c(phi), _c(psi)
    n = c0.size
    cb = np.zeros(n)
    sp = np.zeros(n)
    lib().orc_reduction(_p(c0), _p(phi), _p(psi), float(lam), davis.encode()[0:1], n, _p(cb), _p(sp))
    return cb, sp


def assemble(dim, DPhi1, DPhi2, DPhi3, DS, W, smap, n_q, nnz):
    """Oracle element assembly.  DPhi* shape (n_int, n_p); DS (n_int, ns*ns); smap (n_e, n_ld^2)."""
    DPhi1, DPhi2 = _c(DPhi1), _c(DPhi2)
    DPhi3 = _c(DPhi3) if DPhi3 is not None else None
    DS, W, smap = _c(DS), _c(W), _c(smap, np.int64)
    n_p = DPhi1.shape[1]
    n_e = smap.shape[0]
    V = np.zeros(nnz)
    lib().orc_assemble(dim, _p(DPhi1), _p(DPhi2), _p(DPhi3), _p(DS), _p(W), _p(smap), n_p, n_e, n_q, _p(V))
    return V


# ----------------------------------------------------------------- reference MEX

_ref_libs: dict = {}
_MX_DOUBLE, _MX_INT32, _MX_INT64 = 6, 12, 14


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "constitutive_problem_3D_SDS_mex.so"))


def _ref(name: str) -> C.CDLL:
    if name not in _ref_libs:
        path = os.path.join(REF_DIR, name + ".so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference build missing: {path} (run oracle.native.build())")
        L = C.CDLL(path, mode=os.RTLD_LOCAL | 2)
        L.sgref_call.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_int, C.c_void_p, C.c_void_p]
        L.sgref_call.restype = C.c_int
        L.sgref_last_error.restype = C.c_char_p
        _ref_libs[name] = L
    return _ref_libs[name]


def _mex(name: str, inputs, out_shapes):
    """Run one reference mexFunction.  inputs: list of (array, mx class); arrays are given
    in numpy row-major form whose memory equals the Octave column-major matrix (m x n)
    when numpy shape is (n, m)."""
    L = _ref(name)
    k = len(inputs)
    keep = []
    ptrs = (C.c_void_p * k)()
    cls = (C.c_int * k)()
    ms = (C.c_int64 * k)()
    ns = (C.c_int64 * k)()
    for i, (arr, m, n, c) in enumerate(inputs):
        keep.append(arr)
        ptrs[i] = arr.ctypes.data
        cls[i] = c
        ms[i] = m
        ns[i] = n
    outs = [np.zeros(s) for s in out_shapes]
    optr = (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    olen = (C.c_int64 * len(outs))(*[o.size for o in outs])
    rc = L.sgref_call(k, ptrs, cls, ms, ns, len(outs), optr, olen)
    if rc != 0:
        raise RuntimeError(f"{name}: {L.sgref_last_error().decode()}")
    return outs


def ref_constitutive(dim, E, c_bar, sin_phi, shear, bulk, lame, want_ds=True):
    """Reference MEX constitutive_problem_{2,3}D_{S,SDS}_mex on the same layout as ``constitutive``."""
    E = _c(E)
    n = E.shape[0]
    ns_in = 6 if dim == 3 else 3
    ns_out, nds = (6, 36) if dim == 3 else (4, 9)
    ins = [(E, ns_in, n, _MX_DOUBLE)] + [(_c(x), 1, n, _MX_DOUBLE) for x in (c_bar, sin_phi, shear, bulk, lame)]
    name = f"constitutive_problem_{dim}D_{'SDS' if want_ds else 'S'}_mex"
    shapes = [(n, ns_out)] + ([(n, nds)] if want_ds else [])
    outs = _mex(name, ins, shapes)
    return outs[0], (outs[1] if want_ds else None)


def ref_assemble(dim, DPhi1, DPhi2, DPhi3, DS, W, smap, n_q, nnz):
    """Reference MEX assemble_K_tangent_vals{,_2D}."""
    DPhi1, DPhi2 = _c(DPhi1), _c(DPhi2)
    n_int, n_p = DPhi1.shape
    DS, W, smap = _c(DS), _c(W), _c(smap, np.int64)
    n_e, nl2 = smap.shape
    nq = np.array([n_q], np.int32)
    nz = np.array([nnz], np.int32)
    ins = [(DPhi1, n_p, n_int, _MX_DOUBLE), (DPhi2, n_p, n_int, _MX_DOUBLE)]
    if dim == 3:
        ins.append((_c(DPhi3), n_p, n_int, _MX_DOUBLE))
    ins += [(DS, DS.shape[1], n_int, _MX_DOUBLE), (W, 1, n_int, _MX_DOUBLE),
            (smap, nl2, n_e, _MX_INT64), (nq, 1, 1, _MX_INT32), (nz, 1, 1, _MX_INT32)]
    name = "assemble_K_tangent_vals" if dim == 3 else "assemble_K_tangent_vals_2D"
    return _mex(name, ins, [(nnz,)])[0]

"""Device-resident mesh handle and small helpers around the C ABI.

PyTorch is used only to own device memory and to hand out CUDA stream handles; all
computation goes through libslopegpu.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .fem import Mesh

F64 = torch.float64


def ptr(t):
    """Device (or pinned host) pointer of a tensor, None for None."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def hptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def cur_stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def require_cuda():
    if not torch.cuda.is_available():
        raise _lib.SlopeGPUError("a CUDA device is required (no CPU fallback)")


# Bumped by every DeviceMesh operation that writes matrix values, so that cached products of
# a matrix (A W of the deflation basis) can tell whether the values changed since.
_matrix_generation = [0]


def matrix_generation() -> int:
    return _matrix_generation[0]


def _bump():
    _matrix_generation[0] += 1


class DeviceMesh:
    """Owns an ``sg_mesh``: element data, gradients, weights and sparsity patterns on the GPU.

    Mirrors the one-time part of CONSTITUTIVE (set_element_data, init_K_r_pattern,
    build_scatter_map; +CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m:393-464, 538-635)."""

    def __init__(self, mesh: Mesh, dphi, weight, n_q):
        require_cuda()
        self.mesh = mesh
        self.dim = mesh.dim
        self.n_p, self.n_e = mesh.elem.shape
        self.n_n = mesh.n_n
        self.n_q = int(n_q)
        self.ns = 6 if self.dim == 3 else 3
        elem = np.ascontiguousarray(mesh.elem.T, dtype=np.int32)       # n_p x n_e column-major
        Q = np.ascontiguousarray(mesh.Q.T, dtype=np.uint8)              # dim x n_n column-major
        d = [np.ascontiguousarray(x, dtype=np.float64) for x in dphi]
        w = np.ascontiguousarray(weight, dtype=np.float64)
        h = C.c_void_p()
        _lib.call("sg_mesh_create", self.dim, self.n_p, self.n_q, self.n_n, self.n_e, hptr(elem), hptr(d[0]),
                  hptr(d[1]), hptr(d[2]) if self.dim == 3 else None, hptr(w), hptr(Q), C.byref(h))
        self.handle = h
        sizes = np.zeros(5, np.int64)
        _lib.call("sg_mesh_sizes", h, hptr(sizes))
        self.n_dof, self.n_Q, self.nnz_ref, self.n_blocks, self.n_int = (int(x) for x in sizes)
        b = C.c_void_p()
        _lib.call("sg_mesh_bsr", h, C.byref(b))
        self.bsr = b
        self.bb = self.dim * self.dim
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.mask = torch.from_numpy(Q.reshape(-1).astype(np.float64)).to(self.device)
        self.weight = torch.from_numpy(w).to(self.device)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().sg_mesh_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------ reference-facing views
    def pattern(self):
        """(ref_I, ref_J, transpose_perm), 1-based, Octave find() order."""
        I = np.zeros(self.nnz_ref, np.int64)
        J = np.zeros(self.nnz_ref, np.int64)
        tp = np.zeros(self.nnz_ref, np.int64)
        _lib.call("sg_mesh_pattern", self.handle, hptr(I), hptr(J), hptr(tp))
        return I, J, tp

    def scatter_map(self):
        nl = self.dim * self.n_p
        m = np.zeros((self.n_e, nl * nl), np.int64)
        _lib.call("sg_mesh_scatter_map", self.handle, hptr(m))
        return m

    def free_dofs(self):
        q = np.zeros(self.n_Q, np.int64)
        _lib.call("sg_mesh_free_dofs", self.handle, hptr(q))
        return q

    def to_ref(self, K):
        V = torch.empty(self.nnz_ref, dtype=F64, device=self.device)
        _lib.call("sg_bsr_to_ref_dev", self.handle, ptr(K), ptr(V), cur_stream())
        return V

    # ------------------------------------------------------------ device operators
    def new_dof_vector(self):
        return torch.zeros(self.n_dof, dtype=F64, device=self.device)

    def new_block_values(self):
        return torch.zeros(self.n_blocks * self.bb, dtype=F64, device=self.device)

    def strain(self, U, E):
        _lib.call("sg_strain_dev", self.handle, ptr(U), ptr(E), cur_stream())

    def force(self, S, s_rows, F):
        _lib.call("sg_force_dev", self.handle, ptr(S), int(s_rows), ptr(F), cur_stream())

    @property
    def fused_residual(self):
        """The fused stress-only residual kernel covers P2 tetrahedra."""
        return self.dim == 3 and self.mesh.elem.shape[0] == 10

    def residual(self, U, c_bar, sin_phi, shear, lame, branch, F):
        _lib.call("sg_residual_dev", self.handle, ptr(U), ptr(c_bar), ptr(sin_phi), ptr(shear), ptr(lame),
                  ptr(branch) if branch is not None else None, ptr(F), cur_stream())

    def assemble(self, DS, K):
        _bump()
        _lib.call("sg_assemble_bsr_dev", self.handle, ptr(DS), ptr(K), cur_stream())

    def elastic_ds(self, shear, bulk, DS):
        _bump()
        _lib.call("sg_elastic_ds_dev", self.handle, ptr(shear), ptr(bulk), ptr(DS), cur_stream())

    def symmetrize(self, K, Ks):
        _bump()
        _lib.call("sg_symmetrize_bsr_dev", self.handle, ptr(K), ptr(Ks), cur_stream())

    def kr_blend(self, r, Kel, Kt, Kr):
        _bump()
        _lib.call("sg_kr_blend_dev", self.handle, float(r), ptr(Kel), ptr(Kt), ptr(Kr), cur_stream())

    def assemble_kr(self, DS, r, Kel, Kt_scratch, Kr):
        """K_r = r K_el + (1 - r) K_t with K_t assembled from DS in the same call; on P2
        tetrahedra deterministic and without writing K_t (Kt_scratch is left untouched)."""
        _bump()
        _lib.call("sg_assemble_kr_dev", self.handle, ptr(DS), float(r), ptr(Kel), ptr(Kt_scratch), ptr(Kr),
                  cur_stream())

    @property
    def tangent_fused(self):
        """The fused assembly + blend leaves K_t unwritten on P2 tetrahedra."""
        return self.dim == 3 and self.mesh.elem.shape[0] == 10

    def spmv(self, K, x, y):
        _lib.call("sg_bsr_spmv_dev", self.bsr, ptr(K), ptr(x), ptr(y), cur_stream())


def check_device_status():
    """Raises RuntimeError if a library kernel recorded in the device status word that a
    bounded wait gave up (the matrices it assembled are then incomplete); clears the word."""
    st = C.c_int32(0)
    _lib.call("sg_device_status", 1, C.byref(st))
    if st.value:
        raise RuntimeError(f"slopegpu device status {st.value:#x}: a bulk-staged assembly kernel gave up "
                           "waiting for its copies")


def dot(x, y) -> float:
    out = C.c_double()
    _lib.call("sg_dot_dev", x.numel(), ptr(x), ptr(y), C.byref(out), cur_stream())
    return out.value


def masked_diff_norm(a, b, mask) -> float:
    out = C.c_double()
    _lib.call("sg_masked_diff_norm2_dev", a.numel(), ptr(a), ptr(b), ptr(mask), C.byref(out), cur_stream())
    return float(np.sqrt(out.value))


def axpby(a, x, b, y):
    _lib.call("sg_axpby_dev", y.numel(), float(a), ptr(x), float(b), ptr(y), cur_stream())

"""Device mirror of the reference's CONSTITUTIVE handle class.

Same method names, argument meaning and call order as
+CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m (Beremi/slope_stability_octave), with all per-point and
per-matrix state resident on the GPU:

  reduction(lam)                        CONSTITUTIVE.m:178-200   (Davis A/B/C)
  constitutive_problem_stress(U)        :202-233                 (E = B U; S)
  constitutive_problem_stress_tangent   :235-266                 (E = B U; S, DS)
  build_F()                             :268-285                 (F = B'(w S))
  build_F_all / build_F_reduced         :309-348
  build_F_and_DS_all / _reduced         :466-485
  init_K_r_pattern(Q)                   :393-464                 (elastic K on the pattern)
  build_K_r_QQ_vals(r)                  :515-532                 (returns device K_r values)
  build_K_r_QQ_vals_ref(r)              the same as host (I, J, V) in find() order (drop-in)

Vectors U, F are device tensors of n_dof = dim*n_n entries, node-major (Octave's dim x n_n
column-major layout).  K values live in the mesh's node-block pattern.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import _lib
from .device import DeviceMesh, F64, cur_stream, ptr


class Profiler:
    """Named time accumulators, mirroring +PROFILING/Profiler.m (add_time / add_count)."""

    def __init__(self):
        self.times = {}
        self.counts = {}

    def add_time(self, name, t):
        tot, n = self.times.get(name, (0.0, 0))
        self.times[name] = (tot + t, n + 1)

    def add_count(self, name, c):
        self.counts[name] = self.counts.get(name, 0) + c

    def summary(self):
        return {k: dict(total_s=v[0], calls=v[1]) for k, v in sorted(self.times.items(), key=lambda kv: -kv[1][0])}


class _Timer:
    def __init__(self, prof, name):
        self.prof, self.name = prof, name

    def __enter__(self):
        if self.prof is not None:
            torch.cuda.synchronize()
            self.t = time.perf_counter()

    def __exit__(self, *a):
        if self.prof is not None:
            torch.cuda.synchronize()
            self.prof.add_time(self.name, time.perf_counter() - self.t)


class CONSTITUTIVE:
    def __init__(self, dmesh: DeviceMesh, c0, phi, psi, Davis_type, shear, bulk, lame):
        self.m = dmesh
        self.dim = dmesh.dim
        self.n_strain = dmesh.ns
        self.n_int = dmesh.n_int
        dev = dmesh.device
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        self.c0, self.phi, self.psi = t(c0), t(phi), t(psi)
        self.shear, self.bulk, self.lame = t(shear), t(bulk), t(lame)
        if Davis_type not in ("A", "B", "C"):
            raise ValueError("Davis_type must be 'A', 'B' or 'C'")
        self.Davis_type = Davis_type
        n = self.n_int
        ns = self.n_strain
        self.s_rows = 6 if self.dim == 3 else 4
        self.c_bar = torch.zeros(n, dtype=F64, device=dev)
        self.sin_phi = torch.zeros(n, dtype=F64, device=dev)
        self.E = torch.zeros(n * ns, dtype=F64, device=dev)
        self.S = torch.zeros(n * self.s_rows, dtype=F64, device=dev)
        self.DS = torch.zeros(n * ns * ns, dtype=F64, device=dev)
        self.branch = torch.zeros(n, dtype=torch.uint8, device=dev)
        self.F = torch.zeros(dmesh.n_dof, dtype=F64, device=dev)
        self.pattern_initialized = False
        self.K_el = None
        self.K_t = None
        self.K_r = None
        self.profiler = None
        self.lambda_ = None

    # -------------------------------------------------------------- reduction & stress
    def reduction(self, lam):
        with _Timer(self.profiler, "CONSTITUTIVE.reduction"):
            _lib.call("sg_reduction_dev", ptr(self.c0), ptr(self.phi), ptr(self.psi), float(lam),
                      self.Davis_type.encode(), self.n_int, ptr(self.c_bar), ptr(self.sin_phi), cur_stream())
            self.lambda_ = float(lam)
        return self

    def _constitutive(self, with_ds):
        fn = "sg_constitutive3d_dev" if self.dim == 3 else "sg_constitutive2d_dev"
        _lib.call(fn, ptr(self.E), ptr(self.c_bar), ptr(self.sin_phi), ptr(self.shear), ptr(self.bulk),
                  ptr(self.lame), self.n_int, ptr(self.S), ptr(self.DS) if with_ds else None, ptr(self.branch),
                  cur_stream())

    def potential_energy(self, U):
        """Integrated potential WEIGHT * Psi(B U) at the current reduction (CONSTITUTIVE.m:363-387)."""
        with _Timer(self.profiler, "CONSTITUTIVE.potential"):
            self.m.strain(U, self.E)
            out = C.c_double()
            _lib.call("sg_potential_dev", self.dim, ptr(self.E), ptr(self.c_bar), ptr(self.sin_phi), ptr(self.shear),
                      ptr(self.bulk), ptr(self.lame), ptr(self.m.weight), self.n_int, C.byref(out), cur_stream())
        return out.value

    def constitutive_problem_stress(self, U):
        with _Timer(self.profiler, "CONSTITUTIVE.stress"):
            self.m.strain(U, self.E)
            self._constitutive(False)
        return self

    def constitutive_problem_stress_tangent(self, U):
        with _Timer(self.profiler, "CONSTITUTIVE.stress_tangent"):
            self.m.strain(U, self.E)
            self._constitutive(True)
        return self

    def build_F(self, out=None):
        with _Timer(self.profiler, "CONSTITUTIVE.build_F"):
            F = self.F if out is None else out
            self.m.force(self.S, self.s_rows, F)
        return F.clone() if out is None else F

    def _residual(self, U):
        """F(U) at the current reduction: one fused kernel (strain, stress-only return mapping,
        internal force) on P2 tetrahedra, the three steps otherwise.  The fused path leaves
        E and S unset."""
        if not self.m.fused_residual:
            self.constitutive_problem_stress(U)
            return self.build_F()
        with _Timer(self.profiler, "CONSTITUTIVE.residual"):
            self.m.residual(U, self.c_bar, self.sin_phi, self.shear, self.lame, self.branch, self.F)
        return self.F.clone()

    def build_F_all(self, lam, U):
        self.reduction(lam)
        return self._residual(U)

    def build_F_reduced(self, U):
        return self._residual(U)

    def build_F_and_DS_all(self, lam, U):
        self.reduction(lam)
        self.constitutive_problem_stress_tangent(U)
        return self.build_F()

    def build_F_and_DS_reduced(self, U):
        self.constitutive_problem_stress_tangent(U)
        return self.build_F()

    # -------------------------------------------------------------- stiffness
    def init_K_r_pattern(self, Q=None):
        """Elastic K on the pattern (symmetrised), CONSTITUTIVE.m:413-449.  The pattern itself
        was built with the mesh; Q must be the mesh's free-DOF mask."""
        if Q is not None and not np.array_equal(np.asarray(Q, bool), self.m.mesh.Q):
            raise ValueError("Q differs from the mesh's free-DOF mask")
        ns = self.n_strain
        DS_el = torch.empty(self.n_int * ns * ns, dtype=F64, device=self.m.device)
        self.m.elastic_ds(self.shear, self.bulk, DS_el)
        K = self.m.new_block_values()
        self.m.assemble(DS_el, K)
        self.K_el = self.m.new_block_values()
        self.m.symmetrize(K, self.K_el)
        self.K_t = self.m.new_block_values()
        self.K_r = self.m.new_block_values()
        del DS_el, K
        self.pattern_initialized = True
        return self

    def elastic_K_QQ(self):
        """K_elast(Q, Q) on the device pattern, Dirichlet rows and columns replaced by the
        identity (the matrix the LL scripts solve for the elastic start)."""
        if not self.pattern_initialized:
            self.init_K_r_pattern()
        if getattr(self, "K_elQ", None) is None:
            self.K_elQ = self.m.new_block_values()
            self.m.kr_blend(1.0, self.K_el, self.K_el, self.K_elQ)
        return self.K_elQ

    def build_K_tangent_QQ_vals(self):
        with _Timer(self.profiler, "CONSTITUTIVE.build_K_tangent_QQ_vals"):
            self.m.assemble(self.DS, self.K_t)
        return self.K_t

    def build_K_r_QQ_vals(self, r):
        """K_r = sym(r K_el + (1-r) K_t) on the device pattern (Dirichlet rows identity): the
        tangent assembly and the blend in one call (``sg_assemble_kr_dev``); on P2 tetrahedra
        K_t is not stored on the way (``build_K_tangent_QQ_vals`` assembles it on request)."""
        if not self.pattern_initialized:
            raise _lib.SlopeGPUError("init_K_r_pattern must be called first")
        with _Timer(self.profiler, "CONSTITUTIVE.build_K_tangent_QQ_vals"):
            self.m.assemble_kr(self.DS, r, self.K_el, self.K_t, self.K_r)
        return self.K_r

    def build_K_r_QQ_vals_ref(self, r):
        """Drop-in output of build_K_r_QQ_vals: host (I, J, V), 1-based, find() order."""
        K = self.build_K_r_QQ_vals(r)
        V = self.m.to_ref(K).cpu().numpy()
        I, J, _ = self.m.pattern()
        return I, J, V

    def V_elast_QQ(self):
        return self.m.to_ref(self.K_el).cpu().numpy()

"""ORACLE (test infrastructure): CPU baseline of the reference path on the host cores.

Used only by bench.py (the ``cpu_baseline`` leg and ``--impl reference``).  A full SSR
continuation step of the benchmark workload takes the CPU path minutes to hours, so the
baseline is a bounded sample: every operation of a Newton iteration of
+NEWTON/newton_ind_SSR.m:68-175 is timed once on a slice of the workload's mesh (a few cells
deep, the same spacing and materials), the unit costs are scaled to the full size, and the
step time is their sum weighted by the operation counts of the GPU's timed continuation steps
(``step_seconds``).  The model is calibrated against a measurement: ``measured_steps`` runs
genuine continuation steps of the CPU path (the oracle's drivers with ``HostAMGDFGMRES``) on a
one-cell slice, and bench.py scales the model by the measured / modelled time of that step.

  reference's own compiled C (oracle/_ref, OpenMP on all host threads):
      return mapping S+DS and S        constitutive_problem_3D_{SDS,S}_mex.c
      tangent assembly                 assemble_K_tangent_vals.c (int64 scatter map)
  oracle port (NumPy/SciPy; the reference's Octave/sparsersb/HYPRE layer is not available):
      Davis reduction, E = B U, F = B'(w S), K_r blend + symmetrisation (CONSTITUTIVE.m)
      SpMV, dots/axpys of MGS, deflation projection (dfgmres_solver.m)
      one V-cycle and the numeric re-set-up (SpGEMM smoothing and Galerkin products) of the
      oracle's AMG restatement on the same matrix
"""
from __future__ import annotations

import os
import time

import numpy as np
import scipy.sparse as sp

from . import native
from .amg_ref import Hierarchy, _block_dinv, _init_vec
from .octave_ref import build_B, elastic_DS


def _time(fn, reps=1):
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


def node_adjacency_csr(elem, n_n):
    """Node adjacency of a P2 mesh (nodes sharing an element)."""
    n_p, n_e = elem.shape
    r = np.repeat(elem.T, n_p, axis=1).ravel()
    c = np.tile(elem.T, (1, n_p)).ravel()
    A = sp.coo_matrix((np.ones(r.size, np.int8), (r, c)), shape=(n_n, n_n)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return A


class CPUSample:
    """Unit costs of the reference path on the benchmark workload (host arrays)."""

    def __init__(self, mesh, dphi, weight, n_q, mat, pts, log=print):
        self.dim = mesh.dim
        self.n_q = n_q
        self.mesh, self.dphi, self.weight, self.mat, self.pts = mesh, dphi, weight, mat, pts
        self.threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        t0 = time.perf_counter()
        self.B = build_B(self.dim, mesh.elem, mesh.n_n, dphi)
        Qf = mesh.Q.T.ravel()
        self.q = np.nonzero(Qf)[0]
        self.nQ = self.q.size
        # K(Q,Q) pattern from the node adjacency, scatter map in the reference's form
        A = node_adjacency_csr(mesh.elem, mesh.n_n)
        Kfull = sp.kron(A, np.ones((self.dim, self.dim), np.int8), format="csr")
        KQ = Kfull[self.q][:, self.q].tocsc()
        KQ.sort_indices()
        self.nnz = KQ.nnz
        key = (KQ.indices.astype(np.int64) * self.nQ
               + np.repeat(np.arange(self.nQ, dtype=np.int64), np.diff(KQ.indptr)))   # (row, col) of find()
        order = np.argsort(key)
        free = -np.ones(mesh.n_n * self.dim, np.int64)
        free[self.q] = np.arange(self.nQ)
        nl = self.dim * mesh.elem.shape[0]
        ldof = (self.dim * mesh.elem.T[:, :, None] + np.arange(self.dim)[None, None, :]).reshape(mesh.n_e, nl)
        f = free[ldof]
        rows = np.repeat(f[:, :, None], nl, axis=2)
        cols = np.repeat(f[:, None, :], nl, axis=1)
        ok = (rows >= 0) & (cols >= 0)
        k = rows[ok] * self.nQ + cols[ok]
        pos = np.searchsorted(key[order], k)
        smap = np.zeros((mesh.n_e, nl, nl), np.int64)
        smap[ok] = order[pos] + 1
        self.smap = np.ascontiguousarray(smap.transpose(0, 2, 1).reshape(mesh.n_e, nl * nl))
        del smap, rows, cols, ok, k, pos
        # the elastic K(Q,Q) through the reference's own assembly (values in find() order)
        DS_el = elastic_DS(self.dim, mat["shear"], mat["bulk"])
        d3 = dphi[2] if self.dim == 3 else None
        V = native.ref_assemble(self.dim, dphi[0], dphi[1], d3, DS_el, weight, self.smap, n_q, self.nnz)
        Kc = sp.csc_matrix((V, KQ.indices, KQ.indptr), shape=KQ.shape)
        self.K = ((Kc + Kc.T) / 2).tocsr()
        self.K.sort_indices()
        log(f"cpu sample set-up {time.perf_counter() - t0:.1f}s (n_Q={self.nQ}, nnz={self.nnz})")
        self.amg = None

    def build_amg(self, B_nullspace, fixed, log=print):
        t0 = time.perf_counter()
        Kf = sp.csr_matrix(self.K.shape)  # placeholder to keep memory low
        del Kf
        n = self.mesh.n_n * self.dim
        E = sp.csr_matrix((np.ones(self.nQ), (self.q, np.arange(self.nQ))), shape=(n, self.nQ))
        Kfull = (E @ self.K @ E.T + sp.diags(fixed.astype(float))).tocsr()
        self.amg_matrix = Kfull
        self.amg = Hierarchy(Kfull, B_nullspace, self.dim, fixed=fixed, theta=0.02)
        log(f"cpu AMG restatement built {time.perf_counter() - t0:.1f}s")

    def amg_numeric_resetup(self, A):
        """The numeric part of an AMG re-set-up for new values on the kept aggregates: block
        Jacobi inverses, lambda_max power iteration, P = T - omega D^-1 A T and the Galerkin
        products P' A P, coarsest inverse (SciPy's compiled SpGEMM; the interpreted aggregation
        loop of the restatement is not timed, as the reference's coarsening runs in C)."""
        H = self.amg
        for lev in H.levels:
            if "T" not in lev:
                lev["Ainv"] = np.linalg.inv(A.toarray())
                break
            lev = dict(lev, A=A)
            b = lev["b"]
            lev["Dinv"] = _block_dinv(A, b)
            v = _init_vec(A.shape[0])
            lmax = 1.0
            for _ in range(10):
                w = H.dinv(lev, A @ v)
                lmax = np.linalg.norm(w) or 1.0
                v = w / lmax
            T = lev["T"]
            P = (T - (4.0 / 3.0 / lmax) * H._dinv_mat(lev, A @ T)).tocsr()
            Ac = (P.T @ A @ P).tocsr()
            keep = sp.diags((~lev["dead_next"]).astype(float))
            A = (keep @ Ac @ keep + sp.diags(lev["dead_next"].astype(float))).tocsr()

    def unit_costs(self):
        d = self.pts
        m = self.mat
        n = self.mesh.n_n * self.dim
        U = np.zeros(n)
        U[self.q] = np.random.default_rng(1).normal(size=self.nQ) * 1e-3
        c = {}
        c["reduction"] = _time(lambda: native.reduction(m["c0"], m["phi"], m["psi"], 1.1, "B"))
        c["strain"] = _time(lambda: self.B @ U)
        args = (d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"])
        c["constitutive_SDS"] = _time(lambda: native.ref_constitutive(self.dim, *args, want_ds=True))
        c["constitutive_S"] = _time(lambda: native.ref_constitutive(self.dim, *args, want_ds=False))
        S, DS = native.ref_constitutive(self.dim, *args, want_ds=True)
        ws = (self.weight[:, None] * S[:, :6]).ravel()
        c["force"] = _time(lambda: self.B.T @ ws)
        d3 = self.dphi[2] if self.dim == 3 else None
        c["assembly"] = _time(lambda: native.ref_assemble(self.dim, self.dphi[0], self.dphi[1], d3, DS, self.weight,
                                                          self.smap, self.n_q, self.nnz))
        V = np.random.default_rng(2).normal(size=self.nnz)
        perm = np.random.default_rng(3).permutation(self.nnz)
        c["kr_blend"] = _time(lambda: (0.5 * ((1e-4 * V + (1 - 1e-4) * V) + (1e-4 * V + (1 - 1e-4) * V)[perm])))
        x = np.random.default_rng(4).normal(size=self.nQ)
        c["spmv"] = _time(lambda: self.K @ x, reps=2)
        c["dot"] = _time(lambda: x @ x, reps=3)
        c["axpy"] = _time(lambda: x - 0.5 * x, reps=3)
        if self.amg is not None:
            r = np.random.default_rng(5).normal(size=self.amg_matrix.shape[0])
            c["vcycle"] = _time(lambda: self.amg.vcycle(r))
            c["amg_setup"] = _time(lambda: self.amg_numeric_resetup(self.amg_matrix))
        return c


def step_seconds(c, counts):
    """Modelled seconds of one continuation step from unit costs ``c`` and per-step counts.

    counts: newton (iterations), linear (FGMRES iterations, both solves), damping (stress-only
    evaluations in the line search), deflation (mean basis size), krylov_j (mean Arnoldi
    index).  The AMG re-set-up after each value update (HYPRE's update_values redoes the whole
    set-up) is the restatement's set-up time on the same matrix."""
    nn = counts["newton"]
    lin = counts["linear"]
    n_damp = counts["damping"]
    k = counts["deflation"]
    j = counts["krylov_j"]
    stress_tangent = c["reduction"] + c["strain"] + c["constitutive_SDS"] + c["force"]
    stress_only = c["reduction"] + c["strain"] + c["constitutive_S"] + c["force"]
    linearise = c["assembly"] + c["kr_blend"]
    a_orth = k * (c["spmv"] + k * c["dot"])
    per_krylov = c.get("vcycle", 0.0) + 2 * c["spmv"] + 2 * k * c["dot"] + 2 * (j + 1) * (c["dot"] + c["axpy"])
    amg_setup = c.get("amg_setup", 0.0)
    return nn * (stress_tangent + linearise + stress_only + a_orth + amg_setup) + n_damp * stress_only \
        + lin * per_krylov


class HostAMGDFGMRES:
    """The reference's linear solver on the host cores, for timing genuine CPU continuation
    steps: DFGMRES (dfgmres_solver.m restated as oracle.drivers.dfgmres, MGS Arnoldi) with
    deflation by the A-orthogonalised basis of earlier solutions (DFGMRES.m, A_orthogonalize.m)
    and one V-cycle of the oracle's AMG restatement as preconditioner, set up on the first
    matrix and numerically updated for every later one (the reference re-runs BoomerAMG's set-up
    per value update).  Matrices are K(Q,Q) (SciPy); the AMG works on its embedding into all
    DOFs with identity rows on the Dirichlet DOFs.  ``copy()`` shares the AMG and keeps its own
    basis, like the reference's copies."""

    def __init__(self, q, n_full, Z_full, dim, tol=1e-1, maxit=100, defl_tol=1e-3, shared=None):
        self.q, self.n_full, self.dim = q, n_full, dim
        self.tol, self.maxit, self.defl_tol = tol, maxit, defl_tol
        self.shared = shared if shared is not None else dict(Z=Z_full)
        self.W = np.zeros((q.size, 0))
        self.Wa = self.W
        nQ = q.size
        self.E = sp.csr_matrix((np.ones(nQ), (q, np.arange(nQ))), shape=(n_full, nQ))
        fixed = np.ones(n_full, bool)
        fixed[q] = False
        self.fixed = fixed

    def setup_preconditioner(self, K):
        A = (self.E @ K @ self.E.T + sp.diags(self.fixed.astype(float))).tocsr()
        H = self.shared.get("H")
        if H is None:
            self.shared["H"] = Hierarchy(A, self.shared["Z"], self.dim, fixed=self.fixed, theta=0.02)
        else:
            H.update(A)

    setup_preconditioner_ijv = setup_preconditioner
    update_preconditioner_values = setup_preconditioner

    def A_orthogonalize(self, K):
        from .drivers import a_orthogonalize
        self.Wa = a_orthogonalize(self.W, K, self.defl_tol)[0] if self.W.shape[1] else self.W

    def _M(self, r):
        x = np.zeros(self.n_full)
        x[self.q] = r
        return self.shared["H"].vcycle(x)[self.q]

    def solve(self, K, b):
        from .drivers import dfgmres
        x, it, _ = dfgmres(K, b, self._M, self.Wa, self.maxit, self.tol)
        return x, it

    def expand_deflation_basis(self, v):
        self.W = np.column_stack([self.W, v])

    def copy(self):
        new = HostAMGDFGMRES(self.q, self.n_full, None, self.dim, self.tol, self.maxit, self.defl_tol, self.shared)
        new.W = self.W.copy()
        new.Wa = self.Wa
        return new


def measured_steps(S, params, n_steps=1, log=print):
    """Wall time of genuine SSR continuation steps of the CPU path on the problem ``S``: the
    oracle's drivers (newton_ind_SSR.m, SSR_indirect_continuation.m) on the reference's
    return mapping restated in C (liboracle, OpenMP) and HostAMGDFGMRES, ``n_steps`` accepted
    steps after the init phase (the init phase is not timed).  Returns dict(step_wall_time,
    step_newton_iterations, step_linear_iterations, deflation)."""
    from slope_stability_octave_b200.linear_solvers import near_null_space_elasticity

    from .drivers import OracleConstitutive, SSR_indirect_continuation
    mesh = S.mesh
    cons = OracleConstitutive(mesh, S.dphi, S.weight, S.n_q, S.mat)
    f = np.ascontiguousarray(S.f.T).ravel()
    q = np.nonzero(cons.Q)[0]
    Z = near_null_space_elasticity(mesh.coord, mesh.Q)
    solver = HostAMGDFGMRES(q, f.size, Z, mesh.dim)
    stats = {}
    t0 = time.perf_counter()
    SSR_indirect_continuation(params, cons.Q, f, cons, solver, max_steps_after_init=n_steps, stats=stats)
    log(f"cpu continuation: init + {n_steps} steps in {time.perf_counter() - t0:.1f}s, "
        f"steps {stats['step_wall_time']}")
    stats["deflation"] = solver.W.shape[1]
    return stats

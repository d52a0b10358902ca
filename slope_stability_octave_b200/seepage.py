"""Unconfined seepage on the GPU: the reference's SEEPAGE package above the C ABI.

  penalty_parameters      +SEEPAGE/penalty_parameters_3D.m (including its L34 term, which
                          measures the z-difference of vertices 2 and 4), _2D.m
  heter_conduct           +SEEPAGE/heter_conduct.m
  SeepageSystem           the device operators of seepage_problem_{2D,3D}.m / newton_flow.m:
                          residual and Newton tangent (sg_seepage_system_dev), Bw * field
                          (sg_point_gradient_dev), element saturation (sg_seepage_saturation_dev)
  seepage_problem         +SEEPAGE/seepage_problem_3D.m:1-75 / seepage_problem_2D.m (initial
                          linear solve, Newton, grad_p, mater_sat)
  newton_flow             +SEEPAGE/newton_flow.m:1-186 (damped Newton, deflation basis
                          expanded on accepted steps, stop on the relative update)
  seepage_solver          the DFGMRES + AMG solver of the seepage scripts (set_linear_solver
                          with Q_w and no coordinates: scalar AMG on the pressure nodes)

The pressure lives on all nodes; Dirichlet nodes (Q_w false) carry identity rows in the
device matrices and zeros in the right-hand sides, so every Krylov inner product equals the
reference's K(Q_w, Q_w) formulation.
"""
from __future__ import annotations

import ctypes as C
import time
from types import SimpleNamespace

import numpy as np
import torch

from . import _lib
from .device import F64, DeviceMesh, _bump, cur_stream, masked_diff_norm, ptr
from .linear_solvers import AMG, DFGMRES

GRHO = 9.81


def penalty_parameters(coord, elem):
    """eps per element = grho * (shortest vertex-vertex length) / 2 (penalty_parameters_3D.m,
    penalty_parameters_2D.m).  In 3D the reference's sixth length L34 adds the squared
    z-difference of vertices 2 and 4 instead of 3 and 4; that term is kept as it is."""
    coord = np.asarray(coord, np.float64)
    elem = np.asarray(elem)
    P = [coord[:, elem[i]] for i in range(coord.shape[0] + 1)]
    d = lambda a, b: (P[a] - P[b]) ** 2

    if coord.shape[0] == 3:
        L12 = np.sqrt(d(0, 1)[0] + d(0, 1)[1] + d(0, 1)[2])
        L13 = np.sqrt(d(0, 2)[0] + d(0, 2)[1] + d(0, 2)[2])
        L23 = np.sqrt(d(1, 2)[0] + d(1, 2)[1] + d(1, 2)[2])
        L14 = np.sqrt(d(0, 3)[0] + d(0, 3)[1] + d(0, 3)[2])
        L24 = np.sqrt(d(1, 3)[0] + d(1, 3)[1] + d(1, 3)[2])
        L34 = np.sqrt(d(2, 3)[0] + d(2, 3)[1] + d(1, 3)[2])
        lmin = np.minimum.reduce([L12, L13, L23, L14, L24, L34])
    else:
        L12 = np.sqrt(d(0, 1)[0] + d(0, 1)[1])
        L13 = np.sqrt(d(0, 2)[0] + d(0, 2)[1])
        L23 = np.sqrt(d(1, 2)[0] + d(1, 2)[1])
        lmin = np.minimum.reduce([L12, L13, L23])
    return GRHO * lmin / 2


def heter_conduct(mater, n_q, k):
    """Conductivity per integration point: k(mater + 1) repeated over the element's points."""
    k = np.asarray(k, np.float64).reshape(-1)
    return np.repeat(k[np.asarray(mater, np.int64)], n_q)


class ScalarPattern:
    """The mesh's node adjacency with 1 x 1 blocks, for the pressure systems.  Exposes what
    the AMG and DFGMRES objects read from a DeviceMesh (``bsr``, ``n_dof``, ``device``,
    ``mesh.coord``, ``mesh.Q``)."""

    scalar = True

    def __init__(self, dmesh: DeviceMesh, Q_w):
        self.dmesh = dmesh
        b = C.c_void_p()
        _lib.call("sg_mesh_bsr_scalar", dmesh.handle, C.byref(b))
        self.bsr = b
        self.n_dof = dmesh.n_n
        self.n_blocks = dmesh.n_blocks
        self.device = dmesh.device
        self.mesh = SimpleNamespace(coord=dmesh.mesh.coord, Q=np.asarray(Q_w, bool).reshape(1, -1))

    def spmv(self, K, x, y):
        _lib.call("sg_bsr_spmv_dev", self.bsr, ptr(K), ptr(x), ptr(y), cur_stream())


def seepage_solver(dmesh: DeviceMesh, Q_w, tolerance=1e-6, max_iterations=200, deflation_tolerance=1e-3,
                   mixed=False, **amg_opts):
    """DFGMRES with the scalar AMG V-cycle on the pressure nodes (the seepage scripts'
    DFGMRES_HYPRE_BOOMERAMG solver: tolerance 1e-6, 200 iterations, deflation 1e-3)."""
    pat = ScalarPattern(dmesh, Q_w)
    amg = AMG(pat, mixed=mixed, **amg_opts)
    s = DFGMRES(pat, tolerance, max_iterations, deflation_tolerance, 0, amg=amg)
    s.overlap_update = False
    s.symmetric_operator = False      # the tangent's Bw' E C term is not symmetric
    return s


class SeepageSystem:
    """Device data of one seepage problem on a mesh: basis values, conductivity, penalty,
    Dirichlet mask, Dirichlet pressure and the gradient of the vertical coordinate."""

    def __init__(self, dmesh: DeviceMesh, hat, conduct0, Q_w, grho=GRHO):
        self.dmesh = dmesh
        dev = dmesh.device
        mesh = dmesh.mesh
        self.grho = float(grho)
        self.pattern = ScalarPattern(dmesh, Q_w)
        self.hat = torch.from_numpy(np.ascontiguousarray(np.asarray(hat, np.float64).T)).to(dev)   # n_q x n_p
        self.conduct = torch.from_numpy(np.ascontiguousarray(conduct0, np.float64)).to(dev)
        self.eps = torch.from_numpy(np.ascontiguousarray(penalty_parameters(mesh.coord, mesh.elem))).to(dev)
        self.Q_w = np.asarray(Q_w, bool).reshape(-1)
        self.mask = torch.from_numpy(self.Q_w.astype(np.float64)).to(dev)
        y = torch.from_numpy(np.ascontiguousarray(mesh.coord[1], np.float64)).to(dev)
        self.gy = self.gradient(y)          # q2 = Bw * coord(2, :)'

    def new_node_vector(self):
        return torch.zeros(self.dmesh.n_n, dtype=F64, device=self.dmesh.device)

    def new_values(self):
        return torch.zeros(self.dmesh.n_blocks, dtype=F64, device=self.dmesh.device)

    def system(self, pw, kappa_mode=2, K=None, F=None):
        """(K, F) at pw (K or F may be skipped by passing False)."""
        want_K = K is not False
        want_F = F is not False
        K = (self.new_values() if K is None else K) if want_K else None
        F = (self.new_node_vector() if F is None else F) if want_F else None
        if want_K:
            _bump()      # cached products of an earlier K (A W of the deflation basis) are stale
        _lib.call("sg_seepage_system_dev", self.dmesh.handle, ptr(self.hat), ptr(pw), ptr(self.conduct),
                  ptr(self.eps), ptr(self.gy), self.grho, int(kappa_mode), ptr(self.mask), ptr(K), ptr(F),
                  cur_stream())
        return K, F

    def residual(self, pw, F=None):
        return self.system(pw, 2, K=False, F=F)[1]

    def gradient(self, field):
        """Bw * field per integration point, (n_int, dim)."""
        out = torch.empty((self.dmesh.n_int, self.dmesh.dim), dtype=F64, device=self.dmesh.device)
        _lib.call("sg_point_gradient_dev", self.dmesh.handle, ptr(field), ptr(out), cur_stream())
        return out

    def saturation(self, pw):
        """(element mean pressure, mater_sat) per element."""
        mean = torch.empty(self.dmesh.n_e, dtype=F64, device=self.dmesh.device)
        sat = torch.empty(self.dmesh.n_e, dtype=torch.uint8, device=self.dmesh.device)
        _lib.call("sg_seepage_saturation_dev", self.dmesh.handle, ptr(self.hat), ptr(pw), ptr(self.eps),
                  ptr(mean), ptr(sat), cur_stream())
        return mean, sat.bool()


def _norm(v):
    return masked_diff_norm(v, None, None)


def newton_flow(S: SeepageSystem, pw_init, solver, it_max=50, tol=1e-10, it_damp_max=10, log=None):
    """Damped Newton for the penalised unconfined seepage problem (newton_flow.m:47-186).
    Returns (pw, stats)."""
    pw = pw_init.clone()
    it = 0
    norm_ref = max(1.0, _norm(pw_init))
    stats = dict(iterations=0, linear_iterations=[], alphas=[], rel_updates=[], status="unknown")
    t0 = time.perf_counter()
    K = S.new_values()
    f = S.new_node_vector()
    fa = S.new_node_vector()
    while True:
        it += 1
        S.system(pw, 2, K=K, F=f)
        solver.setup_preconditioner(K)
        solver.A_orthogonalize(K)
        dp, lin_it = solver.solve(K, f)
        criterion = _norm(f)
        alpha, it_damp = 1.0, 0
        while it_damp < it_damp_max:
            it_damp += 1
            S.residual(pw + alpha * dp, F=fa)
            if _norm(fa) < criterion:
                break
            alpha /= 2
        if it_damp >= it_damp_max:
            alpha = 0.0
        pw.add_(dp, alpha=alpha)
        if alpha > 0:
            solver.expand_deflation_basis(dp)
        rel_update = _norm(dp) / norm_ref
        stats["linear_iterations"].append(int(lin_it))
        stats["alphas"].append(alpha)
        stats["rel_updates"].append(rel_update)
        if log:
            log(f"seepage_newton it={it} rel_update={rel_update:.2e} alpha={alpha:.2f} lin_it={lin_it}")
        if rel_update < tol:
            stats["status"] = "converged"
            break
        if np.isnan(rel_update):
            stats["status"] = "nan_update"
            break
        if it > it_max:
            stats["status"] = "max_iterations"
            break
    stats["iterations"] = it
    stats["wall_s"] = time.perf_counter() - t0
    return pw, stats


def seepage_problem(dmesh: DeviceMesh, hat, Q_w, pw_D, conduct0, grho=GRHO, solver=None, it_max=50, tol=1e-10,
                    log=None):
    """[pw, grad_p, mater_sat] of seepage_problem_3D.m / seepage_problem_2D.m on the device.
    pw_D: Dirichlet pressure per node (host or device).  Returns device tensors pw (n_n),
    grad_p (n_int, dim), mater_sat (n_e, bool) and the Newton statistics."""
    S = SeepageSystem(dmesh, hat, conduct0, Q_w, grho)
    if solver is None:
        solver = seepage_solver(dmesh, Q_w, 1e-8, 400, 1e-8)    # local_default_hypre_solver
    pwD = torch.as_tensor(np.asarray(pw_D, np.float64) if not torch.is_tensor(pw_D) else pw_D,
                          dtype=F64).to(dmesh.device)
    # initial right-hand side: 3D includes the gravity head term, 2D does not
    K_D, f = S.system(pwD, 1 if dmesh.dim == 3 else 0)
    solver.setup_preconditioner(K_D)
    solver.A_orthogonalize(K_D)
    pw0, lin0 = solver.solve(K_D, f)
    pw_init = pw0 * S.mask + pwD
    pw, stats = newton_flow(S, pw_init, solver, it_max=it_max, tol=tol, log=log)
    stats["initial_linear_iterations"] = int(lin0)
    grad_p = S.gradient(pw)
    _, sat = S.saturation(pw)
    return pw, grad_p, sat, stats

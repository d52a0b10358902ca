"""ORACLE (test infrastructure): NumPy/SciPy restatement of the Newton and continuation drivers.

Follows Beremi/slope_stability_octave, slope_stability/:
  OracleConstitutive      CONSTITUTIVE.m (reduction, stress, build_F, K_r) on the oracle's
                          C restatement (liboracle) and the SciPy pattern of octave_ref
  DirectSolver            +LINEAR_SOLVERS/DIRECT_BACKSLASH.m (u = A \\ b, no deflation)
  dfgmres                 +LINEAR_SOLVERS/dfgmres_solver.m:1-181 (MGS, H \\ g per step)
  a_orthogonalize         +LINEAR_SOLVERS/A_orthogonalize.m:1-58
  newton                  +NEWTON/newton.m:74-165
  newton_ind_SSR          +NEWTON/newton_ind_SSR.m:68-175
  damping, damping_ALG5   +NEWTON/damping.m, damping_ALG5.m
  init_phase / SSR_indirect_continuation   +CONTINUATION/*.m

Vectors are flat over all dim*n_n DOFs (node-major, Octave's dim x n_n column-major); Q is
the boolean mask of free DOFs in that order.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import native
from .octave_ref import OctavePattern


class OracleConstitutive:
    def __init__(self, mesh, dphi, weight, n_q, mat, davis="B"):
        self.dim = mesh.dim
        self.ns = 6 if self.dim == 3 else 3
        self.n_q = n_q
        self.dphi = dphi
        self.mat = mat
        self.davis = davis
        self.pat = OctavePattern(self.dim, mesh.elem, mesh.n_n, dphi, weight, mesh.Q, mat["shear"], mat["bulk"])
        self.smap = self.pat.scatter_map()
        self.Q = np.zeros(mesh.n_n * self.dim, bool)
        self.Q[self.pat.Q_flat] = True
        self.c_bar = self.sin_phi = None
        self.S = self.DS = None
        self.pattern_initialized = True

    def reduction(self, lam):
        self.c_bar, self.sin_phi = native.reduction(self.mat["c0"], self.mat["phi"], self.mat["psi"], lam, self.davis)

    def _stress(self, U, want_ds):
        E = self.pat.strain(U.reshape(-1, self.dim).T)
        S, DS, _ = native.constitutive(self.dim, E, self.c_bar, self.sin_phi, self.mat["shear"], self.mat["bulk"],
                                       self.mat["lame"], want_ds)
        self.S = S
        if want_ds:
            self.DS = DS

    def build_F(self):
        return self.pat.force(self.S).T.ravel()

    def build_F_all(self, lam, U):
        self.reduction(lam)
        self._stress(U, False)
        return self.build_F()

    def build_F_reduced(self, U):
        self._stress(U, False)
        return self.build_F()

    def build_F_and_DS_all(self, lam, U):
        self.reduction(lam)
        self._stress(U, True)
        return self.build_F()

    def build_F_and_DS_reduced(self, U):
        self._stress(U, True)
        return self.build_F()

    def potential_energy(self, U):
        """CONSTITUTIVE.m:363-387: integrated potential WEIGHT * Psi(B U)."""
        E = self.pat.strain(U.reshape(-1, self.dim).T)
        psi = potential(self.dim, E, self.c_bar, self.sin_phi, self.mat["shear"], self.mat["bulk"],
                        self.mat["lame"])
        return float(self.pat.weight @ psi)

    def elastic_K(self):
        """K_elast(Q, Q) (the elastic values of init_K_r_pattern, CONSTITUTIVE.m:393-464)."""
        n = self.pat.n_Q
        return sp.csc_matrix((self.pat.V_elast, (self.pat.ref_I - 1, self.pat.ref_J - 1)), shape=(n, n))

    def build_K_r_QQ_vals(self, r):
        d3 = self.dphi[2] if self.dim == 3 else None
        Vt = native.assemble(self.dim, self.dphi[0], self.dphi[1], d3, self.DS, self.pat.weight, self.smap, self.n_q,
                             self.pat.nnz)
        V = self.pat.K_r_values(Vt, r)
        n = self.pat.n_Q
        return sp.csc_matrix((V, (self.pat.ref_I - 1, self.pat.ref_J - 1)), shape=(n, n))


class DirectSolver:
    """DIRECT_BACKSLASH: exact solves, deflation ignored."""

    def __init__(self):
        self._lu = None

    def setup_preconditioner(self, K):
        self._lu = spla.splu(K.tocsc())

    setup_preconditioner_ijv = setup_preconditioner
    update_preconditioner_values = setup_preconditioner

    def A_orthogonalize(self, K):
        pass

    def solve(self, K, b):
        return self._lu.solve(b), 0

    def expand_deflation_basis(self, v):
        pass

    def copy(self):
        return DirectSolver()


def a_orthogonalize(W, A, eps_add):
    """A_orthogonalize.m: W (m x n) -> (W_orth, norms)."""
    m, n = W.shape
    Wo = np.zeros((m, n))
    norms = np.ones(n)
    keep = np.zeros(n, bool)
    for i in range(n):
        temp = W[:, n - 1 - i].copy()
        At = A @ temp
        if i > 0:
            temp = temp - (Wo[:, :i] * norms[:i]) @ (At @ Wo[:, :i])
        nt = temp @ At
        if abs(nt) > eps_add:
            if nt > 0:
                nt = math.sqrt(nt)
            else:
                nt = math.sqrt(abs(nt))
                norms[i] = -1
            Wo[:, i] = temp / nt
            keep[i] = True
    Wo, norms = Wo[:, keep], norms[keep]
    return Wo[:, ::-1], norms[::-1]


def dfgmres(A, b, M, W, maxits, tol):
    """dfgmres_solver.m with MGS and per-step least squares (returns x, iters, res_hist)."""
    n = b.size
    x = np.zeros(n)
    if W is not None and W.shape[1] > 0:
        x = W @ (W.T @ b)
        proj = lambda w: w - W @ (W.T @ (A @ w))
    else:
        proj = lambda w: w
    r0 = b - A @ x
    b_norm = np.linalg.norm(b) or 1.0
    res = np.linalg.norm(r0)
    hist = [res / b_norm]
    if hist[0] < tol:
        return x, 0, hist
    V = np.zeros((n, maxits + 1))
    H = np.zeros((maxits + 1, maxits))
    Z = np.zeros((n, maxits))
    V[:, 0] = r0 / res
    g = np.zeros(maxits + 1)
    g[0] = res
    y = np.zeros(0)
    iters = 0
    for j in range(maxits):
        w = proj(M(V[:, j]))
        u = A @ w
        for i in range(j + 1):
            H[i, j] = V[:, i] @ u
            u = u - H[i, j] * V[:, i]
        H[j + 1, j] = np.linalg.norm(u)
        Z[:, j] = w
        iters = j + 1
        if H[j + 1, j] < 1e-14:
            y = np.linalg.lstsq(H[: j + 1, : j + 1], g[: j + 1], rcond=None)[0]
            break
        V[:, j + 1] = u / H[j + 1, j]
        y = np.linalg.lstsq(H[: j + 2, : j + 1], g[: j + 2], rcond=None)[0]
        res = np.linalg.norm(g[: j + 2] - H[: j + 2, : j + 1] @ y)
        hist.append(res / b_norm)
        if hist[-1] < tol:
            break
    x = x + Z[:, :iters] @ y
    return x, iters, hist


# ---------------------------------------------------------------------------- Newton


def _solveQ(solver, K, rhs, Q):
    u = np.zeros(Q.size)
    uq, nit = solver.solve(K, rhs[Q])
    u[Q] = uq
    return u, nit


def damping(it_damp_max, U_it, dU, F, f, cons):
    decrease = (F - f) @ dU
    if math.isnan(decrease) or np.linalg.norm(dU) == np.inf or decrease >= 0:
        return 0.0
    alpha, a_min, a_max, it = 1.0, 0.0, 1.0, 0
    while it < it_damp_max:
        it += 1
        F_a = cons.build_F_reduced(U_it + alpha * dU)
        decrease = (F_a - f) @ dU
        if decrease < 0:
            if alpha == 1:
                break
            a_min = alpha
        else:
            a_max = alpha
        alpha = (a_min + a_max) / 2
    return alpha


def damping_ALG5(it_damp_max, U_it, lambda_it, d_U, d_l, f, criterion, Q, cons):
    if math.isnan(d_l):
        return 0.0
    alpha, it = 1.0, 0
    while True:
        it += 1
        F_a = cons.build_F_all(lambda_it + alpha * d_l, U_it + alpha * d_U)
        crit = np.linalg.norm(F_a[Q] - f[Q])
        if crit >= criterion:
            alpha /= 2
        else:
            break
        if it >= it_damp_max:
            alpha = 0.0
            break
    return alpha


def newton(U_ini, tol, it_newt_max, it_damp_max, r_min, Q, f, cons, solver):
    U = U_ini.copy()
    norm_f = np.linalg.norm(f[Q])
    r, it, flag, compute = r_min, 0, 0, True
    rel = float("nan")
    F = None
    while True:
        it += 1
        if compute:
            F = cons.build_F_and_DS_reduced(U)
            rel = np.linalg.norm(F[Q] - f[Q]) / norm_f
            if rel < tol:
                break
        K = cons.build_K_r_QQ_vals(r)
        solver.setup_preconditioner(K)
        solver.A_orthogonalize(K)
        dU, _ = _solveQ(solver, K, f - F, Q)
        alpha = damping(it_damp_max, U, dU, F, f, cons)
        compute = True
        if alpha < 1e-1:
            if alpha == 0:
                compute = False
                r *= 2
            else:
                r *= 2 ** 0.25
        else:
            solver.expand_deflation_basis(dU[Q])
            if alpha > 0.5:
                r = max(r / math.sqrt(2), r_min)
        if alpha == 0 and r > 1:
            if rel > 10 * tol:
                flag = 1
            break
        U = U + alpha * dU
        if math.isnan(rel) or it == it_newt_max:
            if rel > 10 * tol:
                flag = 1
            break
    return U, flag, it


def newton_ind_SSR(U_ini, omega, lambda_ini, it_newt_max, it_damp_max, tol, r_min, Q, f, cons, solver):
    U = U_ini.copy()
    lam = float(lambda_ini)
    eps = tol / 1000
    fQ = f[Q]
    norm_f = np.linalg.norm(fQ)
    r, it, flag, compute = r_min, 0, 0, True
    rel = float("nan")
    F = criterion = None
    hist = dict(residual=[], lin_W=[], lin_V=[])
    while True:
        it += 1
        if compute:
            F = cons.build_F_and_DS_all(lam, U)
            criterion = np.linalg.norm(F[Q] - fQ)
            rel = criterion / norm_f
            hist["residual"].append(rel)
            if rel < tol and it > 1:
                break
        K = cons.build_K_r_QQ_vals(r)
        F_eps = cons.build_F_all(lam + eps, U)
        G = (F_eps - F) / eps
        solver.setup_preconditioner(K)
        solver.A_orthogonalize(K)
        W, lw = _solveQ(solver, K, -G, Q)
        V, lv = _solveQ(solver, K, f - F, Q)
        hist["lin_W"].append(lw)
        hist["lin_V"].append(lv)
        d_l = -(fQ @ V[Q]) / (fQ @ W[Q])
        d_U = V + d_l * W
        alpha = damping_ALG5(it_damp_max, U, lam, d_U, d_l, f, criterion, Q, cons)
        compute = True
        if alpha < 1e-1:
            if alpha == 0:
                compute = False
                r *= 2
            else:
                r *= 2 ** 0.25
        else:
            solver.expand_deflation_basis(W[Q])
            solver.expand_deflation_basis(V[Q])
            if alpha > 0.5:
                r = max(r / math.sqrt(2), r_min)
        if alpha == 0 and r > 1:
            if rel > 10 * tol:
                flag = 1
            break
        U = U + alpha * d_U
        U = omega * U / (fQ @ U[Q])
        lam = lam + alpha * d_l
        if math.isnan(rel) or it == it_newt_max:
            if rel > 10 * tol:
                flag = 1
            break
    return U, lam, flag, it, hist


def SSR_indirect_continuation(p, Q, f, cons, solver, max_steps_after_init=None, stats=None):
    """p: dict of the continuation parameters (SSR_indirect_continuation.m arguments).
    ``stats`` (optional dict) receives per accepted step its wall time (the sum of its
    attempts, SSR_indirect_continuation.m:186), Newton iterations and linear iterations."""
    import time
    if stats is not None:
        stats.update(step_wall_time=[], step_newton_iterations=[], step_linear_iterations=[])
    wall_acc = lin_acc = it_acc = 0
    fQ = f[Q]
    cons.reduction(p["lambda_init"])
    U1, flag, _ = newton(np.zeros_like(f), p["tol"], p["it_newt_max"], p["it_damp_max"], p["r_min"], Q, f, cons,
                         solver.copy())
    if flag:
        raise RuntimeError("Initial choice of lambda seems to be too large.")
    omega1 = fQ @ U1[Q]
    d_lambda, lambda1 = p["d_lambda_init"], p["lambda_init"]
    solver.expand_deflation_basis(U1[Q])        # init_phase_SSR_indirect_continuation.m:97
    while True:
        lam_it = lambda1 + d_lambda
        cons.reduction(lam_it)
        U_it, flag, _ = newton(U1, p["tol"], p["it_newt_max"], p["it_damp_max"], p["r_min"], Q, f, cons,
                               solver.copy())
        if flag:
            d_lambda /= 2
        else:
            U2, omega2, lambda2 = U_it, fQ @ U_it[Q], lam_it
            if (omega2 - omega1) / max(1, omega1) < 1e-5:
                U1, lambda1, omega1 = U2, lambda2, omega2
            else:
                break
        if d_lambda < p["d_lambda_min"]:
            raise RuntimeError("It seems that the FoS is equal to lambda_init.")
        if lambda1 > 10:
            raise RuntimeError("It seems that the FoS is greater than 10.")
    U_old, U, omega_old, omega, lam = U1, U2, omega1, omega2, lambda2
    solver.expand_deflation_basis(U_old[Q])     # SSR_indirect_continuation.m:85
    lambda_hist, omega_hist = [lambda1, lambda2], [omega1, omega2]
    newton_its = []
    d_omega = omega - omega_old
    step, n_omega, accepted = 2, 0, 0
    while True:
        omega_it = min(omega + d_omega, p["omega_max_stop"])
        d_omega = omega_it - omega
        U_ini = d_omega * (U - U_old) / (omega - omega_old) + U
        t0 = time.perf_counter()
        U_it, lam_it, flag, it, hist = newton_ind_SSR(U_ini, omega_it, lam, p["it_newt_max"], p["it_damp_max"],
                                                      p["tol"], p["r_min"], Q, f, cons, solver.copy())
        wall_acc += time.perf_counter() - t0
        it_acc += it
        lin_acc += sum(hist["lin_W"]) + sum(hist["lin_V"])
        if flag:
            d_omega /= 2
            n_omega += 1
        else:
            step += 1
            U_old, U = U, U_it
            solver.expand_deflation_basis(U[Q])     # SSR_indirect_continuation.m:173
            omega_old, omega = omega, omega_it
            d_lambda = lam_it - lam
            lam = lam_it
            n_omega = 0
            omega_hist.append(omega)
            lambda_hist.append(lam)
            newton_its.append(it)
            accepted += 1
            if stats is not None:
                stats["step_wall_time"].append(wall_acc)
                stats["step_newton_iterations"].append(it_acc)
                stats["step_linear_iterations"].append(lin_acc)
            wall_acc = lin_acc = it_acc = 0
            if (d_lambda / d_omega) * (omega_hist[step - 1] - omega_hist[0]) < p["d_lambda_diff_scaled_min"]:
                break
            if omega >= p["omega_max_stop"]:
                break
            if (lambda_hist[step - 1] - lambda_hist[step - 2]) < 0.9 * (lambda_hist[step - 2] - lambda_hist[step - 3]):
                d_omega *= 2
            if max_steps_after_init is not None and accepted >= max_steps_after_init:
                break
        if n_omega >= 5 or step >= p["step_max"]:
            break
    return np.array(lambda_hist), np.array(omega_hist), newton_its, U


# ---------------------------------------------------------------------------- limit load


def newton_ind_LL(U_ini, t_ini, omega, it_newt_max, it_damp_max, tol, r_min, Q, f, cons, solver):
    """newton_ind_LL.m:55-167: F(U) = t f with f(Q)' U(Q) = omega; returns (U, t, flag, it)."""
    U = U_ini.copy()
    t = float(t_ini)
    fQ = f[Q]
    norm_f = np.linalg.norm(fQ)
    r, it, flag, compute = r_min, 0, 0, True
    F = None
    while True:
        it += 1
        if compute:
            F = cons.build_F_and_DS_reduced(U)
        criterion = np.linalg.norm(F[Q] - t * fQ)
        rel = criterion / norm_f
        if criterion < tol * norm_f and it > 1:
            break
        K = cons.build_K_r_QQ_vals(r)
        solver.setup_preconditioner(K)
        solver.A_orthogonalize(K)
        W, _ = _solveQ(solver, K, f, Q)
        V, _ = _solveQ(solver, K, t * f - F, Q)
        d_t = -(fQ @ V[Q]) / (fQ @ W[Q])
        dU = V + d_t * W
        alpha = damping(it_damp_max, U, dU, F, F * 0, cons)   # newton_ind_LL.m:134 passes f = 0
        compute = True
        if alpha < 1e-1:
            if alpha == 0:
                compute = False
                r *= 2
            else:
                r *= 2 ** 0.25
        else:
            solver.expand_deflation_basis(W[Q])
            solver.expand_deflation_basis(V[Q])
            if alpha > 0.5:
                r = max(r / math.sqrt(2), r_min)
        if alpha == 0 and r > 1:
            flag = 1
            break
        U = U + alpha * dU
        U = omega * U / (fQ @ U[Q])
        t = t + d_t
        if math.isnan(rel) or it == it_newt_max:
            flag = 1
            break
    return U, t, flag, it


def LL_elastic_start(Q, f, cons, solver):
    """The LL scripts' start (slope_stability_3D_homo_LL.m:121-129): elastic solution at
    lambda = 1, omega increment one fifth of its work, U_elast scaled by 1/5."""
    cons.reduction(1.0)
    K = cons.elastic_K()
    solver.setup_preconditioner(K)
    U, _ = _solveQ(solver, K, f, Q)
    solver.expand_deflation_basis(U[Q])
    omega_el = f[Q] @ U[Q]
    return U / 5, omega_el / 5


def LL_indirect_continuation(d_omega_ini, d_t_min, step_max, omega_max, it_newt_max, it_damp_max, tol, r_min,
                             U_elast, Q, f, cons, solver, max_steps=None):
    """LL_indirect_continuation.m:47-158; returns (t_hist, omega_hist, newton_its, U) with the
    reference's leading zero entries."""
    omega = omega_old = 0.0
    d_omega = d_omega_ini
    t = 0.0
    U = U_elast.copy()
    U_old = U.copy()
    U_ini = U.copy()
    n_omega, step, accepted = 0, 1, 0
    t_hist, omega_hist, its = [0.0], [0.0], []
    while True:
        omega_it = omega + d_omega
        if omega_it > omega_max:
            omega_it = omega_max
            d_omega = omega_it - omega
        if step > 1:
            U_ini = d_omega * (U - U_old) / (omega - omega_old) + U
        U_it, t_it, flag, nit = newton_ind_LL(U_ini, t, omega_it, it_newt_max, it_damp_max, tol, r_min, Q, f, cons,
                                              solver.copy())
        if flag == 1:
            d_omega /= 2
            n_omega += 1
        else:
            step += 1
            accepted += 1
            U_old, U = U, U_it
            solver.expand_deflation_basis(U[Q])
            omega_old, omega = omega, omega_it
            d_t = t_it - t
            t = t_it
            n_omega = 0
            omega_hist.append(omega)
            t_hist.append(t)
            its.append(nit)
            if d_t < d_t_min:
                break
            if nit < 20 and step > 2 and (t_hist[step - 1] - t_hist[step - 2]) < 0.9 * (t_hist[step - 2] - t_hist[step - 3]):
                d_omega = 2 * d_omega
            if max_steps is not None and accepted >= max_steps:
                break
        if n_omega >= 5 or omega >= omega_max or step >= step_max:
            break
    return np.array(t_hist), np.array(omega_hist), its, U


# ---------------------------------------------------------------------------- SSR direct


def potential(dim, E, c_bar, sin_phi, shear, bulk, lame):
    """Per-point elastoplastic potential Psi of the trial strain: potential_3D.m:36-123 and
    potential_2D.m:26-95 (E is (n, 6) in 3D, (n, 3) in 2D; engineering shears)."""
    sp = sin_phi
    if dim == 3:
        t = E.copy()
        t[:, 3:] *= 0.5
        I1 = t[:, 0] + t[:, 1] + t[:, 2]
        I2 = t[:, 0] * t[:, 1] + t[:, 0] * t[:, 2] + t[:, 1] * t[:, 2] - t[:, 3] ** 2 - t[:, 4] ** 2 - t[:, 5] ** 2
        I3 = (t[:, 0] * t[:, 1] * t[:, 2] - t[:, 2] * t[:, 3] ** 2 - t[:, 1] * t[:, 5] ** 2 - t[:, 0] * t[:, 4] ** 2
              + 2 * t[:, 3] * t[:, 4] * t[:, 5])
        Q = np.maximum(0.0, (1 / 9) * (I1 ** 2 - 3 * I2))
        R = (1 / 54) * (-2 * I1 ** 3 + 9 * (I1 * I2) - 27 * I3)
        th0 = np.zeros_like(Q)
        pos = Q > 0
        th0[pos] = R[pos] / np.sqrt(Q[pos] ** 3)
        th = np.arccos(np.clip(th0, -1, 1)) / 3
        e1 = -2 * np.sqrt(Q) * np.cos(th + 2 * np.pi / 3) + I1 / 3
        e2 = -2 * np.sqrt(Q) * np.cos(th - 2 * np.pi / 3) + I1 / 3
        e3 = -2 * np.sqrt(Q) * np.cos(th) + I1 / 3
        f_tr = 2 * shear * ((1 + sp) * e1 - (1 - sp) * e3) + 2 * (lame * sp) * I1 - c_bar
        den_s = 4 * lame * sp ** 2 + 4 * shear * (1 + sp ** 2)
    else:
        I1 = E[:, 0] + E[:, 1]
        I2 = np.sqrt((E[:, 0] - E[:, 1]) ** 2 + E[:, 2] ** 2)
        a, b, c = (I1 + I2) / 2, (I1 - I2) / 2, np.zeros_like(I1)
        e1, e2, e3 = a.copy(), b.copy(), c.copy()
        t2 = (a >= c) & (c > b)
        e2[t2], e3[t2] = c[t2], b[t2]
        t3 = c > a
        e1[t3], e2[t3], e3[t3] = c[t3], a[t3], b[t3]
        I1 = e1 + e2 + e3
        f_tr = 2 * shear * ((1 + sp) * e1 - (1 - sp) * e3) + 2 * lame * sp * I1 - c_bar
        den_s = 4 * lame * sp ** 2 + 2 * shear * (1 + sp) ** 2 + 2 * shear * (1 - sp) ** 2
    g_sl = (e1 - e2) / (1 + sp)
    g_sr = (e2 - e3) / (1 - sp)
    g_la = (e1 + e2 - 2 * e3) / (3 - sp)
    g_ra = (2 * e1 - e2 - e3) / (3 + sp)
    den_l = 4 * lame * sp ** 2 + shear * (1 + sp) ** 2 + 2 * shear * (1 - sp) ** 2
    den_r = 4 * lame * sp ** 2 + 2 * shear * (1 + sp) ** 2 + shear * (1 - sp) ** 2
    den_a = 4 * bulk * sp ** 2
    tr = e1 + e2 + e3
    l_s = f_tr / den_s
    l_l = (shear * ((1 + sp) * (e1 + e2) - 2 * (1 - sp) * e3) + 2 * lame * sp * tr - c_bar) / den_l
    l_r = (shear * (2 * (1 + sp) * e1 - (1 - sp) * (e2 + e3)) + 2 * lame * sp * tr - c_bar) / den_r
    l_a = (2 * bulk * sp * tr - c_bar) / den_a
    el_part = 0.5 * lame * tr ** 2
    psi = np.zeros_like(tr)
    t_el = f_tr <= 0
    psi[t_el] = (el_part + shear * (e1 ** 2 + e2 ** 2 + e3 ** 2))[t_el]
    t_s = (l_s <= np.minimum(g_sl, g_sr)) & ~t_el
    psi[t_s] = (el_part + shear * (e1 ** 2 + e2 ** 2 + e3 ** 2) - 0.5 * den_s * l_s ** 2)[t_s]
    t_l = (g_sl < g_sr) & (l_l >= g_sl) & (l_l <= g_la) & ~(t_el | t_s)
    psi[t_l] = (el_part + shear * (e3 ** 2 + 0.5 * (e1 + e2) ** 2) - 0.5 * den_l * l_l ** 2)[t_l]
    t_r = (g_sl > g_sr) & (l_r >= g_sr) & (l_r <= g_ra) & ~(t_el | t_s)
    psi[t_r] = (el_part + shear * (e1 ** 2 + 0.5 * (e2 + e3) ** 2) - 0.5 * den_r * l_r ** 2)[t_r]
    t_a = ~(t_el | t_s | t_l | t_r)
    psi[t_a] = (0.5 * bulk * tr ** 2 - 0.5 * den_a * l_a ** 2)[t_a]
    return psi


def omega_SSR_direct(lambda_ini, U_ini, eps, d_lambda, it_newt_max, it_damp_max, tol, r_min, Q, f, cons, solver):
    """omega_SSR_direct_continuation.m:32-68: U at lambda, omega = dJ/dlambda by a backward
    difference of the energy J = Psi - f'U over eps."""
    cons.reduction(lambda_ini)
    U, flag, _ = newton(U_ini, tol, it_newt_max, it_damp_max, r_min, Q, f, cons, solver)
    if flag:
        return U, 0.0, 1
    J = cons.potential_energy(U) - f[Q] @ U[Q]
    beta = min(1.0, eps / d_lambda)
    U_beta = beta * U_ini + (1 - beta) * U
    cons.reduction(lambda_ini - eps)
    U_eps, flag, _ = newton(U_beta, tol, it_newt_max, it_damp_max, r_min, Q, f, cons, solver)
    if flag:
        return U, 0.0, 1
    J_eps = cons.potential_energy(U_eps) - f[Q] @ U_eps[Q]
    return U, (J_eps - J) / eps, 0


def SSR_direct_continuation(p, Q, f, cons, solver, max_steps_after_init=None):
    """init_phase_SSR_direct_continuation.m + SSR_direct_continuation.m:52-150; returns
    (lambda_hist, omega_hist)."""
    tol = p["tol"]
    eps = tol * 100
    args = (p["it_newt_max"], p["it_damp_max"], tol, p["r_min"], Q, f, cons)
    U1, omega1, flag = omega_SSR_direct(p["lambda_init"], np.zeros_like(f), eps, 1000, *args, solver.copy())
    if flag:
        raise RuntimeError("Initial choice of lambda seems to be too large.")
    d_lambda, lambda1 = p["d_lambda_init"], p["lambda_init"]
    while True:
        lam_it = lambda1 + d_lambda
        solver.expand_deflation_basis(U1[Q])
        U_it, omega_it, flag = omega_SSR_direct(lam_it, U1, eps, d_lambda, *args, solver.copy())
        if flag:
            d_lambda /= 2
        else:
            U2, omega2, lambda2 = U_it, omega_it, lam_it
            if (omega2 - omega1) / max(1, omega1) < 1e-5:
                U1, lambda1, omega1 = U2, lambda2, omega2
            else:
                break
        if d_lambda < p["d_lambda_min"]:
            raise RuntimeError("It seems that FoS is equal to lambda_init.")
        if lambda1 > 10:
            raise RuntimeError("It seems that the FoS is greater than 10.")
    U, omega, lam = U2, omega2, lambda2
    solver.expand_deflation_basis(U[Q])
    lambda_hist, omega_hist = [lambda1, lam], [omega1, omega]
    d_omega = omega - omega1
    d_lambda = lam - p["lambda_init"]
    step, accepted = 2, 0
    while True:
        lam_it = lam + d_lambda
        U_it, omega_it, flag = omega_SSR_direct(lam_it, U, eps, d_lambda, *args, solver.copy())
        d_omega_test = omega_it - omega_hist[step - 1]
        if flag or d_omega_test < 0:
            d_lambda /= 2
        else:
            U, omega, lam = U_it, omega_it, lam_it
            step += 1
            accepted += 1
            lambda_hist.append(lam)
            omega_hist.append(omega)
            solver.expand_deflation_basis(U[Q])
            if (d_lambda / d_omega_test) * (omega_hist[step - 1] - omega_hist[0]) < p["d_lambda_diff_scaled_min"]:
                break
            if d_omega_test > 1.5 * d_omega:
                d_lambda /= 2
            d_omega = d_omega_test
            if max_steps_after_init is not None and accepted >= max_steps_after_init:
                break
        if d_lambda < p["d_lambda_min"] or step >= p["step_max"]:
            break
    return np.array(lambda_hist), np.array(omega_hist)

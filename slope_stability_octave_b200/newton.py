"""Semismooth Newton drivers with regularisation and damping (device mirror of +NEWTON).

  newton          +NEWTON/newton.m:1-192         (fixed lambda; init phase)
  newton_ind_SSR  +NEWTON/newton_ind_SSR.m:1-193 (omega-constrained SSR step: lambda is an unknown)
  newton_ind_LL   +NEWTON/newton_ind_LL.m:1-198  (omega-constrained limit-load step)
  damping         +NEWTON/damping.m:1-56         (bisection on the descent condition)
  damping_ALG5    +NEWTON/damping_ALG5.m:1-60    (halving on the residual norm)

Vectors U, F, f are flat device tensors over all DOFs (node-major); Q is the device mask
(1 free / 0 Dirichlet).  The control flow, tolerances, regularisation updates (r *= 2,
r *= 2^(1/4), r = max(r / sqrt(2), r_min)), deflation-basis expansion and stopping tests
follow the reference statement by statement.
"""
from __future__ import annotations

import math
import time

import torch

from .device import check_device_status, dot, masked_diff_norm


def _norm_masked(x, Q):
    return masked_diff_norm(x, None, Q)


def damping(it_damp_max, U_it, dU, F, f, cons):
    decrease = dot(F, dU) - dot(f, dU)
    ndu = math.sqrt(max(dot(dU, dU), 0.0))
    if math.isnan(decrease) or math.isinf(ndu) or decrease >= 0:
        return 0.0
    alpha, a_min, a_max = 1.0, 0.0, 1.0
    it = 0
    while it < it_damp_max:
        it += 1
        U_alpha = U_it + alpha * dU
        F_alpha = cons.build_F_reduced(U_alpha)
        decrease = dot(F_alpha, dU) - dot(f, dU)
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
    alpha = 1.0
    it = 0
    while True:
        it += 1
        U_alpha = U_it + alpha * d_U
        lam_alpha = lambda_it + alpha * d_l
        F_alpha = cons.build_F_all(lam_alpha, U_alpha)
        crit = masked_diff_norm(F_alpha, f, Q)
        if crit >= criterion:
            alpha = alpha / 2
        else:
            break
        if it >= it_damp_max:
            alpha = 0.0
            break
    return alpha


def newton(U_ini, tol, it_newt_max, it_damp_max, r_min, K_elast, Q, f, cons, solver, verbose=False):
    U_it = U_ini.clone()
    fQ = f * Q
    norm_f = _norm_masked(f, Q)
    r = r_min
    it = 0
    flag = 0
    compute_diffs = True
    if not cons.pattern_initialized:
        cons.init_K_r_pattern()
    hist = dict(residual=[], r=[], alpha=[], linear_iters=[])
    rel_resid = float("nan")
    status = "unknown"
    ijv_init = False
    t0 = time.perf_counter()
    F = None
    while True:
        it += 1
        if compute_diffs:
            F = cons.build_F_and_DS_reduced(U_it)
            criterion = masked_diff_norm(F, f, Q)
            rel_resid = criterion / norm_f
            hist["residual"].append(rel_resid)
            if rel_resid < tol:
                status = "converged"
                break
        hist["r"].append(r)
        K = cons.build_K_r_QQ_vals(r)
        if not ijv_init:
            solver.setup_preconditioner_ijv(K)
            ijv_init = True
        else:
            solver.update_preconditioner_values(K)
        solver.A_orthogonalize(K)
        b = fQ - F * Q
        dU, lin_it = solver.solve(K, b)
        hist["linear_iters"].append(lin_it)
        alpha = damping(it_damp_max, U_it, dU, F, f, cons)
        hist["alpha"].append(alpha)
        compute_diffs = True
        if alpha < 1e-1:
            if alpha == 0:
                compute_diffs = False
                r = r * 2
            else:
                r = r * 2 ** 0.25
        else:
            solver.expand_deflation_basis(dU)
            if alpha > 0.5:
                r = max(r / math.sqrt(2), r_min)
        if alpha == 0 and r > 1:
            status = "stalled_regularization"
            if rel_resid > 10 * tol:
                flag = 1
            break
        U_it = U_it + alpha * dU
        if verbose:
            print(f"  newton it={it} rel_resid={rel_resid:.2e} alpha={alpha:.2f} r={r:.3g} lin_it={lin_it}")
        if math.isnan(rel_resid) or it == it_newt_max:
            if rel_resid > 10 * tol:
                flag = 1
            status = "nan_residual" if math.isnan(rel_resid) else "max_iterations"
            break
    hist["status"] = status
    hist["wall_time"] = time.perf_counter() - t0
    hist["linear_iters_total"] = int(sum(hist["linear_iters"]))
    check_device_status()
    return U_it, flag, it, hist


def newton_ind_SSR(U_ini, omega, lambda_ini, it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons, solver,
                   verbose=False):
    U_it = U_ini.clone()
    lambda_it = float(lambda_ini)
    eps = tol / 1000
    fQ = f * Q
    norm_f = _norm_masked(f, Q)
    flag = 0
    compute_diffs = True
    r = r_min
    it = 0
    hist = dict(residual=[], r=[], alpha=[], linear_iters_W=[], linear_iters_V=[])
    rel_resid = float("nan")
    status = "unknown"
    if not cons.pattern_initialized:
        cons.init_K_r_pattern()
    ijv_init = False
    t0 = time.perf_counter()
    F = None
    criterion = None
    while True:
        it += 1
        if compute_diffs:
            F = cons.build_F_and_DS_all(lambda_it, U_it)
            criterion = masked_diff_norm(F, f, Q)
            rel_resid = criterion / norm_f
            hist["residual"].append(rel_resid)
            if rel_resid < tol and it > 1:
                status = "converged"
                break
        hist["r"].append(r)
        K = cons.build_K_r_QQ_vals(r)
        # the preconditioner update is issued before the residual at lambda + eps (the
        # reference computes F_eps first; neither depends on the other), so that the two,
        # and the A-orthogonalisation, overlap when the update runs on a side stream
        if not ijv_init:
            solver.setup_preconditioner_ijv(K)
            ijv_init = True
        else:
            solver.update_preconditioner_values(K)
        F_eps = cons.build_F_all(lambda_it + eps, U_it)
        G = (F_eps - F) / eps
        solver.A_orthogonalize(K)
        # the two systems are independent: solved side by side when the solver can
        (W, lin_w), (V, lin_v) = solver.solve_pair(K, -G * Q, fQ - F * Q)
        hist["linear_iters_W"].append(lin_w)
        hist["linear_iters_V"].append(lin_v)
        d_l = -dot(fQ, V) / dot(fQ, W)
        d_U = V + d_l * W
        alpha = damping_ALG5(it_damp_max, U_it, lambda_it, d_U, d_l, f, criterion, Q, cons)
        hist["alpha"].append(alpha)
        compute_diffs = True
        if alpha < 1e-1:
            if alpha == 0:
                compute_diffs = False
                r = r * 2
            else:
                r = r * 2 ** 0.25
        else:
            solver.expand_deflation_basis(W)
            solver.expand_deflation_basis(V)
            if alpha > 0.5:
                r = max(r / math.sqrt(2), r_min)
        if alpha == 0 and r > 1:
            status = "stalled_regularization"
            if rel_resid > 10 * tol:
                flag = 1
            break
        U_it = U_it + alpha * d_U
        U_it = omega * U_it / dot(fQ, U_it)
        lambda_it = lambda_it + alpha * d_l
        if verbose:
            print(f"  newton_ind_SSR it={it} rel_resid={rel_resid:.2e} alpha={alpha:.2f} r={r:.3g} "
                  f"lin_it=[W:{lin_w},V:{lin_v}] lambda={lambda_it:.8f}")
        if math.isnan(rel_resid) or it == it_newt_max:
            if rel_resid > 10 * tol:
                flag = 1
            status = "nan_residual" if math.isnan(rel_resid) else "max_iterations"
            break
    hist["status"] = status
    hist["wall_time"] = time.perf_counter() - t0
    hist["linear_iters_W_total"] = int(sum(hist["linear_iters_W"]))
    hist["linear_iters_V_total"] = int(sum(hist["linear_iters_V"]))
    check_device_status()
    return U_it, lambda_it, flag, it, hist


def newton_ind_LL(U_ini, t_ini, omega, it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons, solver,
                  verbose=False):
    """F(U) = t f with f(Q)' U(Q) = omega fixed (+NEWTON/newton_ind_LL.m:55-167).  Returns
    (U, t, flag, it, hist)."""
    U_it = U_ini.clone()
    t_it = float(t_ini)
    fQ = f * Q
    norm_f = _norm_masked(f, Q)
    flag = 0
    compute_diffs = True
    r = r_min
    it = 0
    if not cons.pattern_initialized:
        cons.init_K_r_pattern()
    hist = dict(residual=[], r=[], alpha=[], linear_iters_W=[], linear_iters_V=[])
    rel_resid = float("nan")
    status = "unknown"
    ijv_init = False
    t0 = time.perf_counter()
    F = None
    while True:
        it += 1
        if compute_diffs:
            F = cons.build_F_and_DS_reduced(U_it)
        criterion = masked_diff_norm(F, t_it * f, Q)
        rel_resid = criterion / norm_f
        hist["residual"].append(rel_resid)
        if criterion < tol * norm_f and it > 1:
            status = "converged"
            break
        hist["r"].append(r)
        K = cons.build_K_r_QQ_vals(r)
        if not ijv_init:
            solver.setup_preconditioner_ijv(K)
            ijv_init = True
        else:
            solver.update_preconditioner_values(K)
        solver.A_orthogonalize(K)
        (W, lin_w), (V, lin_v) = solver.solve_pair(K, fQ, t_it * fQ - F * Q)
        hist["linear_iters_W"].append(lin_w)
        hist["linear_iters_V"].append(lin_v)
        d_t = -dot(fQ, V) / dot(fQ, W)
        dU = V + d_t * W
        # newton_ind_LL.m:134 passes F_int * 0 as the load of the line search
        alpha = damping(it_damp_max, U_it, dU, F, torch.zeros_like(F), cons)
        hist["alpha"].append(alpha)
        compute_diffs = True
        if alpha < 1e-1:
            if alpha == 0:
                compute_diffs = False
                r = r * 2
            else:
                r = r * 2 ** 0.25
        else:
            solver.expand_deflation_basis(W)
            solver.expand_deflation_basis(V)
            if alpha > 0.5:
                r = max(r / math.sqrt(2), r_min)
        if alpha == 0 and r > 1:
            status = "stalled_regularization"
            flag = 1
            break
        U_it = U_it + alpha * dU
        U_it = omega * U_it / dot(fQ, U_it)
        t_it = t_it + d_t
        if verbose:
            print(f"  newton_ind_LL it={it} rel_resid={rel_resid:.2e} alpha={alpha:.2f} r={r:.3g} "
                  f"lin_it=[W:{lin_w},V:{lin_v}] t={t_it:.8f}")
        if math.isnan(rel_resid) or it == it_newt_max:
            flag = 1
            status = "nan_residual" if math.isnan(rel_resid) else "max_iterations"
            break
    hist["status"] = status
    hist["wall_time"] = time.perf_counter() - t0
    hist["linear_iters_W_total"] = int(sum(hist["linear_iters_W"]))
    hist["linear_iters_V_total"] = int(sum(hist["linear_iters_V"]))
    check_device_status()
    return U_it, t_it, flag, it, hist

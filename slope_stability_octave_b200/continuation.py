"""Indirect SSR continuation (device mirror of +CONTINUATION).

  init_phase_SSR_indirect_continuation   +CONTINUATION/init_phase_SSR_indirect_continuation.m:1-143
  SSR_indirect_continuation              +CONTINUATION/SSR_indirect_continuation.m:1-237

The per-step statistics follow SSR_indirect_continuation.m:53-72,134-195: one accepted step
is the sum of its attempts' wall times (``step_wall_time``), which is the benchmark metric.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from .device import dot
from .newton import newton, newton_ind_SSR


class ContinuationError(RuntimeError):
    pass


def init_phase_SSR_indirect_continuation(lambda_init, d_lambda_init, d_lambda_min, it_newt_max, it_damp_max, tol,
                                         r_min, K_elast, Q, f, cons, solver, verbose=False):
    fQ = f * Q
    U_ini = torch.zeros_like(f)
    if not cons.pattern_initialized:
        cons.init_K_r_pattern()
    cons.reduction(lambda_init)
    its = []
    U_it, flag, it, _ = newton(U_ini, tol, it_newt_max, it_damp_max, r_min, K_elast, Q, f, cons, solver, verbose)
    its.append(it)
    if flag == 1:
        raise ContinuationError("Initial choice of lambda seems to be too large.")
    U1 = U_it
    omega1 = dot(fQ, U1)
    d_lambda = d_lambda_init
    lambda1 = lambda_init
    solver.expand_deflation_basis(U_it)
    while True:
        lambda_it = lambda1 + d_lambda
        cons.reduction(lambda_it)
        U_it, flag, it, _ = newton(U1, tol, it_newt_max, it_damp_max, r_min, K_elast, Q, f, cons, solver, verbose)
        its.append(it)
        if flag == 1:
            d_lambda = d_lambda / 2
        else:
            U2 = U_it
            omega2 = dot(fQ, U2)
            lambda2 = lambda_it
            if (omega2 - omega1) / max(1, omega1) < 1e-5:
                U1, lambda1, omega1 = U2, lambda2, omega2
            else:
                break
        if d_lambda < d_lambda_min:
            raise ContinuationError("It seems that the FoS is equal to lambda_init.")
        if lambda1 > 10:
            raise ContinuationError("It seems that the FoS is greater than 10.")
    return U1, U2, omega1, omega2, lambda1, lambda2, its


def SSR_indirect_continuation(lambda_init, d_lambda_init, d_lambda_min, d_lambda_diff_scaled_min, step_max,
                              omega_max_stop, it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons, solver,
                              verbose=False, max_steps_after_init=None, on_step=None):
    """Returns (U, lambda_hist, omega_hist, Umax_hist, stats).  ``max_steps_after_init``
    optionally stops after that many accepted continuation steps (bounded benchmarks)."""
    t_total = time.perf_counter()
    fQ = f * Q
    stats = dict(init_newton_iterations=[], attempt_step=[], attempt_success=[], attempt_wall_time=[],
                 attempt_newton_iterations=[], attempt_newton_flag=[], attempt_newton_relres_end=[],
                 attempt_omega_target=[], attempt_lambda_before=[], attempt_lambda_after=[],
                 attempt_linear_iterations=[], step_index=[], step_attempt_count=[], step_wall_time=[],
                 step_newton_iterations=[], step_newton_iterations_total=[], step_newton_relres_end=[],
                 step_lambda=[], step_omega=[], step_linear_iterations=[])
    t_init = time.perf_counter()
    U_old, U, omega_old, omega, lambda_old, lam, its = init_phase_SSR_indirect_continuation(
        lambda_init, d_lambda_init, d_lambda_min, it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons,
        solver.copy(), verbose)
    stats["init_wall_time"] = time.perf_counter() - t_init
    stats["init_newton_iterations"] = its
    solver.expand_deflation_basis(U_old)
    lambda_hist = [lambda_old, lam]
    omega_hist = [omega_old, omega]
    umax = lambda V: float(torch.sqrt((V.reshape(-1, cons.dim) ** 2).sum(1)).max())
    Umax_hist = [umax(U_old), umax(U)]
    d_omega = omega - omega_old
    if omega_max_stop < omega + d_omega:
        raise ContinuationError("Too small value of omega_max_stop.")
    step = 2
    n_omega, n_omega_max = 0, 5
    wall_acc, it_acc, cnt_acc, lin_acc = 0.0, 0, 0, 0
    n_accepted = 0
    stop_reason = ""
    while True:
        omega_it = min(omega + d_omega, omega_max_stop)
        d_omega = omega_it - omega
        U_ini = d_omega * (U - U_old) / (omega - omega_old) + U
        torch.cuda.synchronize()
        t_att = time.perf_counter()
        U_it, lambda_it, flag, it_newt, hist = newton_ind_SSR(U_ini, omega_it, lam, it_newt_max, it_damp_max, tol,
                                                              r_min, K_elast, Q, f, cons, solver.copy(), verbose)
        torch.cuda.synchronize()
        att_wall = time.perf_counter() - t_att
        relres = hist["residual"][-1] if hist["residual"] else float("nan")
        lin_total = hist["linear_iters_W_total"] + hist["linear_iters_V_total"]
        stats["attempt_step"].append(step + 1)
        stats["attempt_success"].append(flag == 0)
        stats["attempt_wall_time"].append(att_wall)
        stats["attempt_newton_iterations"].append(it_newt)
        stats["attempt_newton_flag"].append(flag)
        stats["attempt_newton_relres_end"].append(relres)
        stats["attempt_omega_target"].append(omega_it)
        stats["attempt_lambda_before"].append(lam)
        stats["attempt_lambda_after"].append(lambda_it if flag == 0 else float("nan"))
        stats["attempt_linear_iterations"].append(lin_total)
        wall_acc += att_wall
        it_acc += it_newt
        cnt_acc += 1
        lin_acc += lin_total
        if verbose:
            print(f"Step {step + 1}: omega={omega_it:.6g} flag={flag} lambda={lambda_it:.8f} newton_it={it_newt} "
                  f"lin_it={lin_total} wall={att_wall:.3f}s")
        if flag == 1:
            d_omega = d_omega / 2
            n_omega += 1
        else:
            step += 1
            U_old, U = U, U_it
            solver.expand_deflation_basis(U)
            omega_old, omega = omega, omega_it
            d_lambda = lambda_it - lam
            lam = lambda_it
            n_omega = 0
            omega_hist.append(omega)
            lambda_hist.append(lam)
            Umax_hist.append(umax(U))
            stats["step_index"].append(step)
            stats["step_attempt_count"].append(cnt_acc)
            stats["step_wall_time"].append(wall_acc)
            stats["step_newton_iterations"].append(it_newt)
            stats["step_newton_iterations_total"].append(it_acc)
            stats["step_newton_relres_end"].append(relres)
            stats["step_lambda"].append(lam)
            stats["step_omega"].append(omega)
            stats["step_linear_iterations"].append(lin_acc)
            wall_acc, it_acc, cnt_acc, lin_acc = 0.0, 0, 0, 0
            n_accepted += 1
            if on_step is not None:
                on_step(step, lam, omega)
            if (d_lambda / d_omega) * (omega_hist[step - 1] - omega_hist[0]) < d_lambda_diff_scaled_min:
                stop_reason = "minimal increase of lambda"
                break
            if omega >= omega_max_stop:
                stop_reason = "maximal omega"
                break
            if (lambda_hist[step - 1] - lambda_hist[step - 2]) < 0.9 * (lambda_hist[step - 2] - lambda_hist[step - 3]):
                d_omega = 2 * d_omega
            if max_steps_after_init is not None and n_accepted >= max_steps_after_init:
                stop_reason = "step budget"
                break
        if n_omega >= n_omega_max:
            stop_reason = "impossible to increase omega"
            break
        if step >= step_max:
            stop_reason = "maximal number of steps"
            break
    stats["stop_reason"] = stop_reason
    stats["total_wall_time"] = time.perf_counter() - t_total
    return U, np.array(lambda_hist), np.array(omega_hist), np.array(Umax_hist), stats

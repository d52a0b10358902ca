"""Indirect SSR and limit-load continuation (device mirror of +CONTINUATION).

  init_phase_SSR_indirect_continuation   +CONTINUATION/init_phase_SSR_indirect_continuation.m:1-143
  SSR_indirect_continuation              +CONTINUATION/SSR_indirect_continuation.m:1-237
  LL_elastic_start                       the LL scripts' start, slope_stability_3D_homo_LL.m:121-129
  LL_indirect_continuation               +CONTINUATION/LL_indirect_continuation.m:1-160
  omega_SSR_direct_continuation          +CONTINUATION/omega_SSR_direct_continuation.m:1-68
  init_phase_SSR_direct_continuation     +CONTINUATION/init_phase_SSR_direct_continuation.m:1-110
  SSR_direct_continuation                +CONTINUATION/SSR_direct_continuation.m:1-150

``SSRIndirectStepper`` is the same loop split into ``init()`` and ``step()`` (one accepted
continuation step per call, including its rejected attempts), so that a caller can time,
checkpoint or drive individual steps; ``SSR_indirect_continuation`` runs it to the end.
The per-step statistics follow SSR_indirect_continuation.m:53-72,134-195: one accepted step
is the sum of its attempts' wall times (``step_wall_time``), which is the benchmark metric.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .device import dot
from .newton import newton, newton_ind_LL, newton_ind_SSR


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


class SSRIndirectStepper:
    """SSR_indirect_continuation.m split into init() and step().  Parameters as the reference
    function (``p`` holds lambda_init, d_lambda_init, d_lambda_min, d_lambda_diff_scaled_min,
    step_max, omega_max_stop, it_newt_max, it_damp_max, tol, r_min)."""

    def __init__(self, p, Q, f, cons, solver, K_elast=None, verbose=False):
        self.p, self.Q, self.f, self.cons, self.solver = dict(p), Q, f, cons, solver
        self.K_elast = K_elast
        self.verbose = verbose
        self.fQ = f * Q
        self.stats = dict(init_newton_iterations=[], attempt_step=[], attempt_success=[], attempt_wall_time=[],
                          attempt_newton_iterations=[], attempt_newton_flag=[], attempt_newton_relres_end=[],
                          attempt_omega_target=[], attempt_lambda_before=[], attempt_lambda_after=[],
                          attempt_linear_iterations=[], step_index=[], step_attempt_count=[], step_wall_time=[],
                          step_newton_iterations=[], step_newton_iterations_total=[], step_newton_relres_end=[],
                          step_lambda=[], step_omega=[], step_linear_iterations=[])
        self.finished = False
        self.stop_reason = ""

    def _umax(self, V):
        return float(torch.sqrt((V.reshape(-1, self.cons.dim) ** 2).sum(1)).max())

    def init(self):
        p = self.p
        t0 = time.perf_counter()
        (self.U_old, self.U, self.omega_old, self.omega, lambda_old, self.lam, its) = \
            init_phase_SSR_indirect_continuation(p["lambda_init"], p["d_lambda_init"], p["d_lambda_min"],
                                                 p["it_newt_max"], p["it_damp_max"], p["tol"], p["r_min"],
                                                 self.K_elast, self.Q, self.f, self.cons, self.solver.copy(),
                                                 self.verbose)
        self.stats["init_wall_time"] = time.perf_counter() - t0
        self.stats["init_newton_iterations"] = its
        self.solver.expand_deflation_basis(self.U_old)
        self.lambda_hist = [lambda_old, self.lam]
        self.omega_hist = [self.omega_old, self.omega]
        self.Umax_hist = [self._umax(self.U_old), self._umax(self.U)]
        self.d_omega = self.omega - self.omega_old
        if p["omega_max_stop"] < self.omega + self.d_omega:
            raise ContinuationError("Too small value of omega_max_stop.")
        self.step_no = 2
        self.n_omega = 0
        return self

    # step-control state besides U, U_old and the deflation basis
    _STATE = ("omega", "omega_old", "lam", "d_omega", "step_no", "n_omega", "finished", "stop_reason")

    def snapshot(self):
        """The continuation's state after its last accepted step: U and U_old (device copies),
        the step-control scalars, the lambda/omega/Umax histories and the solver's deflation
        basis.  ``restore(snapshot)`` puts the run back there (checkpoint/resume; a benchmark
        replays the continuation from a fixed point)."""
        return dict(U=self.U.clone(), U_old=self.U_old.clone(), basis=self.solver.basis.clone(),
                    state={k: getattr(self, k) for k in self._STATE},
                    hist=(list(self.lambda_hist), list(self.omega_hist), list(self.Umax_hist)))

    def restore(self, snap):
        """Continue from a ``snapshot()``: the next step() repeats the step that followed it.
        The statistics keep accumulating."""
        self.U = snap["U"].clone()
        self.U_old = snap["U_old"].clone()
        for k, v in snap["state"].items():
            setattr(self, k, v)
        self.lambda_hist, self.omega_hist, self.Umax_hist = (list(h) for h in snap["hist"])
        self.solver.basis = snap["basis"].clone()
        self.solver.AW, self.solver._aw_key = None, None
        return self

    def step(self):
        """Attempts until one is accepted (or the run stops).  Returns the accepted step's
        statistics, or None if the continuation stopped without accepting a step."""
        p, st = self.p, self.stats
        wall_acc, it_acc, cnt_acc, lin_acc = 0.0, 0, 0, 0
        while not self.finished:
            omega_it = min(self.omega + self.d_omega, p["omega_max_stop"])
            self.d_omega = omega_it - self.omega
            U_ini = self.d_omega * (self.U - self.U_old) / (self.omega - self.omega_old) + self.U
            torch.cuda.synchronize()
            t_att = time.perf_counter()
            U_it, lambda_it, flag, it_newt, hist = newton_ind_SSR(
                U_ini, omega_it, self.lam, p["it_newt_max"], p["it_damp_max"], p["tol"], p["r_min"], self.K_elast,
                self.Q, self.f, self.cons, self.solver.copy(), self.verbose)
            torch.cuda.synchronize()
            att_wall = time.perf_counter() - t_att
            relres = hist["residual"][-1] if hist["residual"] else float("nan")
            lin_total = hist["linear_iters_W_total"] + hist["linear_iters_V_total"]
            st["attempt_step"].append(self.step_no + 1)
            st["attempt_success"].append(flag == 0)
            st["attempt_wall_time"].append(att_wall)
            st["attempt_newton_iterations"].append(it_newt)
            st["attempt_newton_flag"].append(flag)
            st["attempt_newton_relres_end"].append(relres)
            st["attempt_omega_target"].append(omega_it)
            st["attempt_lambda_before"].append(self.lam)
            st["attempt_lambda_after"].append(lambda_it if flag == 0 else float("nan"))
            st["attempt_linear_iterations"].append(lin_total)
            wall_acc += att_wall
            it_acc += it_newt
            cnt_acc += 1
            lin_acc += lin_total
            if self.verbose:
                print(f"Step {self.step_no + 1}: omega={omega_it:.6g} flag={flag} lambda={lambda_it:.8f} "
                      f"newton_it={it_newt} lin_it={lin_total} wall={att_wall:.3f}s")
            accepted = None
            if flag == 1:
                self.d_omega = self.d_omega / 2
                self.n_omega += 1
            else:
                self.step_no += 1
                step = self.step_no
                self.U_old, self.U = self.U, U_it
                self.solver.expand_deflation_basis(self.U)
                self.omega_old, self.omega = self.omega, omega_it
                d_lambda = lambda_it - self.lam
                self.lam = lambda_it
                self.n_omega = 0
                self.omega_hist.append(self.omega)
                self.lambda_hist.append(self.lam)
                self.Umax_hist.append(self._umax(self.U))
                accepted = dict(step=step, wall=wall_acc, attempts=cnt_acc, newton_iterations=it_newt,
                                newton_iterations_total=it_acc, linear_iterations=lin_acc, relres=relres,
                                lam=self.lam, omega=self.omega)
                st["step_index"].append(step)
                st["step_attempt_count"].append(cnt_acc)
                st["step_wall_time"].append(wall_acc)
                st["step_newton_iterations"].append(it_newt)
                st["step_newton_iterations_total"].append(it_acc)
                st["step_newton_relres_end"].append(relres)
                st["step_lambda"].append(self.lam)
                st["step_omega"].append(self.omega)
                st["step_linear_iterations"].append(lin_acc)
                lh, oh = self.lambda_hist, self.omega_hist
                if (d_lambda / self.d_omega) * (oh[step - 1] - oh[0]) < p["d_lambda_diff_scaled_min"]:
                    self.finished, self.stop_reason = True, "minimal increase of lambda"
                elif self.omega >= p["omega_max_stop"]:
                    self.finished, self.stop_reason = True, "maximal omega"
                elif (lh[step - 1] - lh[step - 2]) < 0.9 * (lh[step - 2] - lh[step - 3]):
                    self.d_omega = 2 * self.d_omega
            if self.n_omega >= 5:
                self.finished, self.stop_reason = True, "impossible to increase omega"
            elif self.step_no >= p["step_max"]:
                self.finished, self.stop_reason = True, "maximal number of steps"
            if accepted is not None:
                return accepted
        return None


def SSR_indirect_continuation(lambda_init, d_lambda_init, d_lambda_min, d_lambda_diff_scaled_min, step_max,
                              omega_max_stop, it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons, solver,
                              verbose=False, max_steps_after_init=None, on_step=None):
    """Returns (U, lambda_hist, omega_hist, Umax_hist, stats).  ``max_steps_after_init``
    optionally stops after that many accepted continuation steps (bounded benchmarks)."""
    t_total = time.perf_counter()
    p = dict(lambda_init=lambda_init, d_lambda_init=d_lambda_init, d_lambda_min=d_lambda_min,
             d_lambda_diff_scaled_min=d_lambda_diff_scaled_min, step_max=step_max, omega_max_stop=omega_max_stop,
             it_newt_max=it_newt_max, it_damp_max=it_damp_max, tol=tol, r_min=r_min)
    run = SSRIndirectStepper(p, Q, f, cons, solver, K_elast, verbose).init()
    n = 0
    while not run.finished:
        acc = run.step()
        if acc is None:
            break
        n += 1
        if on_step is not None:
            on_step(acc["step"], acc["lam"], acc["omega"])
        if max_steps_after_init is not None and n >= max_steps_after_init:
            run.stop_reason = "step budget"
            break
    st = run.stats
    st["stop_reason"] = run.stop_reason
    st["total_wall_time"] = time.perf_counter() - t_total
    return run.U, np.array(run.lambda_hist), np.array(run.omega_hist), np.array(run.Umax_hist), st


def LL_elastic_start(Q, f, cons, solver):
    """Elastic solution at lambda = 1 as the start of the limit-load continuation: returns
    (U_elast / 5, omega_el / 5) with omega_el = f(Q)' U_elast(Q) (the LL scripts' set-up,
    slope_stability_3D_homo_LL.m:121-129); the solution joins the deflation basis."""
    cons.reduction(1.0)
    K = cons.elastic_K_QQ()
    solver.setup_preconditioner(K)
    U, _ = solver.solve(K, f * Q)
    solver.expand_deflation_basis(U)
    omega_el = dot(f * Q, U)
    return U / 5, omega_el / 5


def LL_indirect_continuation(d_omega_ini, d_t_min, step_max, omega_max, it_newt_max, it_damp_max, tol, r_min,
                             K_elast, U_elast, Q, f, cons, solver, verbose=False, max_steps=None):
    """Returns (U, t_hist, omega_hist, Umax_hist, stats); the histories start with the
    reference's leading zero entry.  ``max_steps`` optionally stops after that many accepted
    steps (bounded runs)."""
    t_total = time.perf_counter()
    omega = omega_old = 0.0
    d_omega = float(d_omega_ini)
    t = 0.0
    U = U_elast.clone()
    U_old = U.clone()
    U_ini = U.clone()
    n_omega, step, accepted = 0, 1, 0
    t_hist, omega_hist, umax_hist = [0.0], [0.0], [0.0]
    stats = dict(step_newton_iterations=[], step_wall_time=[], step_linear_iterations=[], attempts=[])
    attempts, wall = 0, 0.0
    stop = ""
    dim = cons.dim
    while True:
        omega_it = omega + d_omega
        if omega_it > omega_max:
            omega_it = omega_max
            d_omega = omega_it - omega
        if step > 1:
            U_ini = d_omega * (U - U_old) / (omega - omega_old) + U
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        U_it, t_it, flag, nit, hist = newton_ind_LL(U_ini, t, omega_it, it_newt_max, it_damp_max, tol, r_min,
                                                    K_elast, Q, f, cons, solver.copy(), verbose)
        torch.cuda.synchronize()
        wall += time.perf_counter() - t0
        attempts += 1
        if flag == 1:
            d_omega = d_omega / 2
            n_omega += 1
        else:
            step += 1
            accepted += 1
            U_old, U = U, U_it
            solver.expand_deflation_basis(U)
            omega_old, omega = omega, omega_it
            d_t = t_it - t
            t = t_it
            n_omega = 0
            omega_hist.append(omega)
            t_hist.append(t)
            umax_hist.append(float(torch.sqrt((U.reshape(-1, dim) ** 2).sum(1)).max()))
            stats["step_newton_iterations"].append(nit)
            stats["step_wall_time"].append(wall)
            stats["step_linear_iterations"].append(hist["linear_iters_W_total"] + hist["linear_iters_V_total"])
            stats["attempts"].append(attempts)
            attempts, wall = 0, 0.0
            if verbose:
                print(f"  accepted: t={t:.8g} d_t={d_t:.6g} omega={omega:.6g} newton_it={nit}")
            if d_t < d_t_min:
                stop = "minimal increment of t"
                break
            if nit < 20 and step > 2 and (t_hist[step - 1] - t_hist[step - 2]) < 0.9 * (t_hist[step - 2] - t_hist[step - 3]):
                d_omega = 2 * d_omega
            if max_steps is not None and accepted >= max_steps:
                stop = "step budget"
                break
        if n_omega >= 5:
            stop = "impossible to increase omega further"
            break
        if omega >= omega_max:
            stop = "maximal omega"
            break
        if step >= step_max:
            stop = "maximal number of steps"
            break
    stats["stop_reason"] = stop
    stats["total_wall_time"] = time.perf_counter() - t_total
    return U, np.array(t_hist), np.array(omega_hist), np.array(umax_hist), stats


def omega_SSR_direct_continuation(lambda_ini, U_ini, eps, d_lambda, it_newt_max, it_damp_max, tol, r_min, K_elast, Q,
                                  f, cons, solver, verbose=False):
    """U at strength reduction lambda and omega = dJ/dlambda, J = Psi(U) - f(Q)'U(Q), by a
    backward difference over eps (+CONTINUATION/omega_SSR_direct_continuation.m:32-68).
    Returns (U, omega, flag); omega = 0 when a Newton solve failed (flag 1)."""
    fQ = f * Q
    cons.reduction(lambda_ini)
    U, flag, _, _ = newton(U_ini, tol, it_newt_max, it_damp_max, r_min, K_elast, Q, f, cons, solver, verbose)
    if flag == 1:
        return U, 0.0, 1
    J = cons.potential_energy(U) - dot(fQ, U)
    beta = min(1.0, eps / d_lambda)
    U_beta = beta * U_ini + (1 - beta) * U
    cons.reduction(lambda_ini - eps)
    U_eps, flag, _, _ = newton(U_beta, tol, it_newt_max, it_damp_max, r_min, K_elast, Q, f, cons, solver, verbose)
    if flag == 1:
        return U, 0.0, 1
    J_eps = cons.potential_energy(U_eps) - dot(fQ, U_eps)
    return U, (J_eps - J) / eps, 0


def init_phase_SSR_direct_continuation(lambda_init, d_lambda_init, d_lambda_min, it_newt_max, it_damp_max, tol, eps,
                                       r_min, K_elast, Q, f, cons, solver, verbose=False):
    """+CONTINUATION/init_phase_SSR_direct_continuation.m:43-110: the first two points."""
    args = (it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons)
    U1, omega1, flag = omega_SSR_direct_continuation(lambda_init, torch.zeros_like(f), eps, 1000, *args,
                                                     solver.copy(), verbose)
    if flag == 1:
        raise ContinuationError("Initial choice of lambda seems to be too large.")
    d_lambda, lambda1 = d_lambda_init, lambda_init
    while True:
        lambda_it = lambda1 + d_lambda
        solver.expand_deflation_basis(U1)
        U_it, omega_it, flag = omega_SSR_direct_continuation(lambda_it, U1, eps, d_lambda, *args, solver.copy(),
                                                             verbose)
        if flag == 1:
            d_lambda = d_lambda / 2
        else:
            U2, omega2, lambda2 = U_it, omega_it, lambda_it
            if (omega2 - omega1) / max(1, omega1) < 1e-5:
                U1, lambda1, omega1 = U2, lambda2, omega2
            else:
                break
        if d_lambda < d_lambda_min:
            raise ContinuationError("It seems that FoS is equal to lambda_init.")
        if lambda1 > 10:
            raise ContinuationError("It seems that the FoS is greater than 10.")
    return U1, U2, omega1, omega2, lambda1, lambda2


def SSR_direct_continuation(lambda_init, d_lambda_init, d_lambda_min, d_lambda_diff_scaled_min, step_max,
                            it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons, solver, verbose=False,
                            max_steps_after_init=None):
    """+CONTINUATION/SSR_direct_continuation.m:52-150 (lambda is the control parameter, omega is
    measured).  Returns (U, lambda_hist, omega_hist, Umax_hist, work_hist, stats)."""
    t_total = time.perf_counter()
    eps = tol * 100
    dim = cons.dim
    umax = lambda V: float(torch.sqrt((V.reshape(-1, dim) ** 2).sum(1)).max())
    U_old, U, omega_old, omega, lambda_old, lam = init_phase_SSR_direct_continuation(
        lambda_init, d_lambda_init, d_lambda_min, it_newt_max, it_damp_max, tol, eps, r_min, K_elast, Q, f, cons,
        solver, verbose)
    solver.expand_deflation_basis(U)
    lambda_hist, omega_hist = [lambda_old, lam], [omega_old, omega]
    Umax_hist = [umax(U), umax(U)]
    work_hist = [dot(U_old, f), dot(U, f)]
    d_omega = omega - omega_old
    d_lambda = lam - lambda_init
    step, accepted = 2, 0
    stats = dict(step_wall_time=[], attempts=[])
    attempts, wall = 0, 0.0
    stop = ""
    args = (it_newt_max, it_damp_max, tol, r_min, K_elast, Q, f, cons)
    while True:
        lambda_it = lam + d_lambda
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        U_it, omega_it, flag = omega_SSR_direct_continuation(lambda_it, U, eps, d_lambda, *args, solver.copy(),
                                                             verbose)
        torch.cuda.synchronize()
        wall += time.perf_counter() - t0
        attempts += 1
        d_omega_test = omega_it - omega_hist[step - 1]
        if flag == 1 or d_omega_test < 0:
            d_lambda = d_lambda / 2
        else:
            U, omega, lam = U_it, omega_it, lambda_it
            step += 1
            accepted += 1
            lambda_hist.append(lam)
            omega_hist.append(omega)
            Umax_hist.append(umax(U))
            work_hist.append(dot(U, f))
            solver.expand_deflation_basis(U)
            stats["step_wall_time"].append(wall)
            stats["attempts"].append(attempts)
            attempts, wall = 0, 0.0
            if verbose:
                print(f"  accepted: lambda={lam:.8g} d_lambda={d_lambda:.6g} omega={omega:.6g}")
            if (d_lambda / d_omega_test) * (omega_hist[step - 1] - omega_hist[0]) < d_lambda_diff_scaled_min:
                stop = "minimal increase of lambda"
                break
            if d_omega_test > 1.5 * d_omega:
                d_lambda = d_lambda / 2
            d_omega = d_omega_test
            if max_steps_after_init is not None and accepted >= max_steps_after_init:
                stop = "step budget"
                break
        if d_lambda < d_lambda_min:
            stop = "minimal increment of lambda"
            break
        if step >= step_max:
            stop = "maximal number of steps"
            break
    stats["stop_reason"] = stop
    stats["total_wall_time"] = time.perf_counter() - t_total
    return U, np.array(lambda_hist), np.array(omega_hist), np.array(Umax_hist), np.array(work_hist), stats

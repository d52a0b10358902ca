"""Generate ssr_oracle.npz, ssr_direct_oracle.npz and ll_oracle.npz: the oracle's SSR
(indirect and direct) and limit-load (LL) continuation histories.

    python tests/golden/make_continuation_golden.py [ssr] [ll] [direct] [full]   (default: all four)

The oracle (oracle/drivers.py, a NumPy restatement of SSR_indirect_continuation.m,
newton_ind_SSR.m, newton.m and damping_ALG5.m driving the reference's own compiled return
mapping and assembly) runs with a sparse direct solver, so lambda and omega carry no Krylov or
AMG error.  Cases (three accepted steps after the two-step init phase):

  slope2d the 2D homogeneous slope at h = 0.5 (mesh_P2_2D(0.5, 15, 10, 15, 10, 10)),
          parameters of slope_stability_2D_homo_SSR.m
  small3d the 3D homogeneous slope mesh_P2_3D(N_h = 1, 15, 10, 15, 10, 10, z = 1),
          parameters of slope_stability_3D_homo_SSR.m
  layered3d the same mesh with the four horizontal material layers of the heterogeneous
          slope (problems.slope_3d_layered), parameters of slope_stability_3D_homo_SSR.m
          (indirect continuation only)
SSR direct continuation (SSR_direct_continuation.m with omega from the potential energy,
four accepted steps after the init phase) on the same two meshes, and, for
LL_indirect_continuation.m / newton_ind_LL.m (seven accepted steps from the scripts'
elastic start), the same two meshes with the parameters of slope_stability_{2D,3D}_homo_LL.m,
and (rf3d) the small 3D mesh with lognormal random-field strength
(problems.slope_3d_random_field, seed 20261203) and the 3D LL parameters.
``full`` (ssr_full_oracle.npz): the SSR indirect continuation of slope2d (the 2D homogeneous
slope at h = 0.5, slope_stability_2D_homo_SSR.m's parameters) and of small3d run to the
reference's own stop tests (SSR_indirect_continuation.m:203-211), so the last lambda is the
factor of safety.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.drivers import (DirectSolver, LL_elastic_start, LL_indirect_continuation,  # noqa: E402
                            OracleConstitutive, SSR_direct_continuation, SSR_indirect_continuation)
from slope_stability_octave_b200 import problems  # noqa: E402

STEPS = 3


def cases():
    return {
        "slope2d": (lambda: problems.slope_2d(0.5), problems.SSR_2D),
        "small3d": (lambda: problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 1)), problems.SSR_3D),
    }


def layered_cases():
    return {"layered3d": (lambda: problems.slope_3d_layered(1, dims=(15, 10, 15, 10, 10, 1)), problems.SSR_3D)}


def run_case(make, params, steps=STEPS):
    P = make()
    cons = OracleConstitutive(P.mesh, P.dphi, P.weight, P.n_q, P.mat)
    f = np.ascontiguousarray(P.f.T).ravel()
    lh, oh, its, _ = SSR_indirect_continuation(params, cons.Q, f, cons, DirectSolver(), max_steps_after_init=steps)
    return np.asarray(lh), np.asarray(oh), np.asarray(its, np.int64)


LL_STEPS = 7


def ll_cases():
    return {
        "slope2d": (lambda: problems.slope_2d(0.5), problems.LL_2D),
        "small3d": (lambda: problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 1)), problems.LL_3D),
        # lognormal random-field strength (per-point c and phi) on the same small mesh
        "rf3d": (lambda: problems.slope_3d_random_field(1, dims=(15, 10, 15, 10, 10, 1), seed=20261203),
                 problems.LL_3D),
    }


def run_ll_case(make, p, steps=LL_STEPS):
    P = make()
    cons = OracleConstitutive(P.mesh, P.dphi, P.weight, P.n_q, P.mat)
    f = np.ascontiguousarray(P.f.T).ravel()
    solver = DirectSolver()
    U0, d_omega = LL_elastic_start(cons.Q, f, cons, solver)
    th, oh, its, _ = LL_indirect_continuation(d_omega, p["d_t_min"], p["step_max"], p["omega_max"], p["it_newt_max"],
                                              p["it_damp_max"], p["tol"], p["r_min"], U0, cons.Q, f, cons,
                                              solver.copy(), max_steps=steps)
    return th, oh, np.asarray(its, np.int64)


DIRECT_STEPS = 4


def run_direct_case(make, params, steps=DIRECT_STEPS):
    P = make()
    cons = OracleConstitutive(P.mesh, P.dphi, P.weight, P.n_q, P.mat)
    f = np.ascontiguousarray(P.f.T).ravel()
    return SSR_direct_continuation(params, cons.Q, f, cons, DirectSolver(), max_steps_after_init=steps)


def full_cases():
    return cases()


def main(sections=("ssr", "ll", "direct", "full")):
    out = {}
    for name, (make, params) in ({**cases(), **layered_cases()}.items() if "ssr" in sections else ()):
        t0 = time.perf_counter()
        lh, oh, its = run_case(make, params)
        out[f"{name}_lambda"], out[f"{name}_omega"], out[f"{name}_newton"] = lh, oh, its
        print(name, f"{time.perf_counter() - t0:.1f}s", "lambda", lh, "omega", oh, "newton", its)
    if out:
        np.savez(os.path.join(HERE, "ssr_oracle.npz"), **out)
    out = {}
    for name, (make, params) in (ll_cases().items() if "ll" in sections else ()):
        t0 = time.perf_counter()
        th, oh, its = run_ll_case(make, params)
        out[f"{name}_t"], out[f"{name}_omega"], out[f"{name}_newton"] = th, oh, its
        print("LL", name, f"{time.perf_counter() - t0:.1f}s", "t", th, "omega", oh, "newton", its)
    if out:
        np.savez(os.path.join(HERE, "ll_oracle.npz"), **out)
    out = {}
    for name, (make, params) in (cases().items() if "direct" in sections else ()):
        t0 = time.perf_counter()
        lh, oh = run_direct_case(make, params)
        out[f"{name}_lambda"], out[f"{name}_omega"] = lh, oh
        print("direct", name, f"{time.perf_counter() - t0:.1f}s", "lambda", lh, "omega", oh)
    if out:
        np.savez(os.path.join(HERE, "ssr_direct_oracle.npz"), **out)
    out = {}
    for name, (make, params) in (full_cases().items() if "full" in sections else ()):
        t0 = time.perf_counter()
        lh, oh, its = run_case(make, params, steps=None)
        out[f"{name}_lambda"], out[f"{name}_omega"], out[f"{name}_newton"] = lh, oh, its
        print("full", name, f"{time.perf_counter() - t0:.1f}s", "steps", its.size, "FoS", lh[-1], "newton", its)
    if out:
        np.savez(os.path.join(HERE, "ssr_full_oracle.npz"), **out)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("ssr", "ll", "direct", "full"))

"""Generate ssr_oracle.npz: the oracle's SSR indirect continuation histories.

    python tests/golden/make_continuation_golden.py

The oracle (oracle/drivers.py, a NumPy restatement of SSR_indirect_continuation.m,
newton_ind_SSR.m, newton.m and damping_ALG5.m driving the reference's own compiled return
mapping and assembly) runs with a sparse direct solver, so lambda and omega carry no Krylov or
AMG error.  Cases (three accepted steps after the two-step init phase):

  cfg0    the 2D homogeneous slope at h = 0.5 (mesh_P2_2D(0.5, 15, 10, 15, 10, 10)),
          parameters of slope_stability_2D_homo_SSR.m
  small3d the 3D homogeneous slope mesh_P2_3D(N_h = 1, 15, 10, 15, 10, 10, z = 1),
          parameters of slope_stability_3D_homo_SSR.m
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.drivers import DirectSolver, OracleConstitutive, SSR_indirect_continuation  # noqa: E402
from slope_stability_octave_b200 import problems  # noqa: E402

STEPS = 3


def cases():
    return {
        "cfg0": (lambda: problems.slope_2d(0.5), problems.SSR_2D),
        "small3d": (lambda: problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 1)), problems.SSR_3D),
    }


def run_case(make, params, steps=STEPS):
    P = make()
    cons = OracleConstitutive(P.mesh, P.dphi, P.weight, P.n_q, P.mat)
    f = np.ascontiguousarray(P.f.T).ravel()
    lh, oh, its, _ = SSR_indirect_continuation(params, cons.Q, f, cons, DirectSolver(), max_steps_after_init=steps)
    return np.asarray(lh), np.asarray(oh), np.asarray(its, np.int64)


def main():
    out = {}
    for name, (make, params) in cases().items():
        t0 = time.perf_counter()
        lh, oh, its = run_case(make, params)
        out[f"{name}_lambda"], out[f"{name}_omega"], out[f"{name}_newton"] = lh, oh, its
        print(name, f"{time.perf_counter() - t0:.1f}s", "lambda", lh, "omega", oh, "newton", its)
    np.savez(os.path.join(HERE, "ssr_oracle.npz"), **out)


if __name__ == "__main__":
    main()

"""Seepage on the GPU (sg_seepage_system_dev, sg_point_gradient_dev, sg_seepage_saturation_dev,
the scalar AMG + DFGMRES) against the oracle (oracle/seepage_ref.py) and the reference's
stored Franz dam run.

  * residual and Newton tangent at pressures that cover the three pieces of the relative
    permeability (negative, inside the penalty band, saturated), for the three right-hand
    side forms, on the 3D slope and the 2D Franz dam mesh: F and K x within 1e-12 of the
    oracle's sparse operators (relative to the largest entry of the oracle's result);
    Bw * pw per point and the element mean pressure within 1e-12, saturation flags equal;
  * the whole seepage problem (initial linear solve, damped Newton, tolerance 1e-10) with the
    GPU Krylov solver at 1e-10: pressure within 1e-8 of the oracle's direct-solve result,
    equal Newton iteration counts and saturation flags, 3D slope and Franz dam (6 Newton
    iterations, as in the stored run);
  * the seepage-coupled SSR continuation on the Franz dam: lambda and omega within 1e-6 of
    the oracle's (direct solves) with equal Newton counts at linear tolerance 1e-10, and, with
    the stored run's own solver settings (seepage DFGMRES 1e-6, mechanics 1e-1), omega_init and
    the lambda of the accepted steps within 1e-4 of the values printed by
    slope_stability_2D_Franz_dam_SSR.ipynb.
"""
import os

import numpy as np
import pytest
import torch

from oracle import seepage_ref as sr
from slope_stability_octave_b200 import continuation, fem, problems, seepage
from slope_stability_octave_b200.device import DeviceMesh

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(__file__), "golden", "seepage_oracle.npz")


def _slope3d():
    mesh = fem.mesh_p2_3d(1, 15, 10, 15, 10, 10, 1)
    xi, wf = fem.quadrature_p2_tet()
    hat, d1, d2, d3 = fem.local_basis_p2_tet(xi)
    D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
    Q_w, pw_D = problems.homo_slope_seepage_bc(mesh.coord)
    return mesh, hat, (D1, D2, D3), W, wf.size, Q_w, pw_D, np.ones(mesh.n_e * wf.size)


def _franz():
    g = np.load(G)
    coord, elem, surf = fem.mesh_p2_from_p1_2d(g["franz_coord_p1"].T, g["franz_elem_p1"].T)
    mater = g["franz_mat"] - 1
    Q = np.ones((2, coord.shape[1]), bool)
    mesh = fem.Mesh(coord, elem, Q)
    xi, wf = fem.quadrature_p2_tri()
    hat, d1, d2 = fem.local_basis_p2_tri(xi)
    D1, D2, W = fem.geometry_2d(mesh, d1, d2, wf)
    Q_w, pw_D = problems.franz_dam_seepage_bc(coord, surf)
    conduct = np.repeat(np.asarray(problems.FRANZ_DAM_K)[mater], wf.size)
    return mesh, hat, (D1, D2), W, wf.size, Q_w, pw_D, conduct


CASES = {"slope3d": _slope3d, "franz_dam": _franz}


@pytest.mark.parametrize("case", sorted(CASES))
def test_seepage_operators_match_oracle(cuda_device, case):
    mesh, hat, dphi, W, n_q, Q_w, pw_D, conduct = CASES[case]()
    dm = DeviceMesh(mesh, dphi, W, n_q)
    S = seepage.SeepageSystem(dm, hat, conduct, Q_w)
    dim = mesh.dim
    Bw, Cm, w = sr.auxiliary_matrices(mesh.elem, dphi, W, hat)
    eps_int = np.repeat(sr.penalty_parameters(mesh.coord, mesh.elem), n_q)
    wc = w * conduct
    import scipy.sparse as sp
    K_D = (Bw.T @ sp.diags(np.repeat(wc, dim)) @ Bw).tocsr()
    q2 = Bw @ mesh.coord[1]
    gq = Bw @ (sr.GRHO * mesh.coord[1])
    rng = np.random.default_rng(7)
    scale = float(np.max(np.abs(pw_D))) or 100.0
    # pressures across the three pieces of perm_r: negative, 0 < p < eps, saturated
    pw = pw_D + rng.uniform(-0.2, 0.6, mesh.n_n) * scale
    pw[rng.random(mesh.n_n) < 0.3] = rng.uniform(0.0, 2.0 * float(eps_int.max()), 1)[0]
    pw_t = torch.from_numpy(pw).cuda()
    mask = Q_w.astype(float)
    for mode in (0, 1, 2):
        K, F = S.system(pw_t, mode)
        K_o, f_o = sr.system(pw, Bw, Cm, K_D, wc, w, conduct, q2, eps_int, sr.GRHO, dim, kappa_mode=mode, gq=gq)
        f_o = f_o * mask
        assert np.max(np.abs(F.cpu().numpy() - f_o)) <= 1e-12 * np.max(np.abs(f_o))
        for _ in range(3):
            x = rng.standard_normal(mesh.n_n) * mask
            y = torch.empty(mesh.n_n, dtype=torch.float64, device="cuda")
            S.pattern.spmv(K, torch.from_numpy(x).cuda(), y)
            y_o = (K_o @ x) * mask
            assert np.max(np.abs(y.cpu().numpy() - y_o)) <= 1e-12 * np.max(np.abs(y_o))
    gp = S.gradient(pw_t).cpu().numpy()
    gp_o = (Bw @ pw).reshape(-1, dim)
    assert np.max(np.abs(gp - gp_o)) <= 1e-12 * np.max(np.abs(gp_o))
    mean, sat = S.saturation(pw_t)
    pint = Cm @ pw
    aver = (pint * w).reshape(mesh.n_e, n_q).sum(1) / w.reshape(mesh.n_e, n_q).sum(1)
    assert np.max(np.abs(mean.cpu().numpy() - aver)) <= 1e-12 * np.max(np.abs(aver))
    eps = sr.penalty_parameters(mesh.coord, mesh.elem)
    decided = np.abs(aver - 0.1 * eps) > 1e-9 * np.abs(aver).max()
    assert np.array_equal(sat.cpu().numpy()[decided], (aver >= 0.1 * eps)[decided])


def test_seepage_problem_matches_oracle_slope3d(cuda_device):
    g = np.load(G)
    mesh, hat, dphi, W, n_q, Q_w, pw_D, conduct = _slope3d()
    dm = DeviceMesh(mesh, dphi, W, n_q)
    solver = seepage.seepage_solver(dm, Q_w, tolerance=1e-10, max_iterations=500)
    pw, grad_p, sat, st = seepage.seepage_problem(dm, hat, Q_w, pw_D, conduct, solver=solver)
    pw = pw.cpu().numpy()
    assert st["status"] == "converged"
    assert st["iterations"] == int(g["homo3d_newton"])
    assert np.max(np.abs(pw - g["homo3d_pw"])) <= 1e-8 * np.max(np.abs(g["homo3d_pw"]))
    assert np.array_equal(sat.cpu().numpy(), g["homo3d_sat"])


def _franz_problem(seepage_tol, maxit):
    g = np.load(G)
    return g, problems.franz_dam(g["franz_coord_p1"], g["franz_elem_p1"], g["franz_mat"],
                                 solver_opts=dict(tolerance=seepage_tol, max_iterations=maxit))


def _ssr(P, tol, steps):
    P.to_device()
    solver = P.solver("DFGMRES_B200", tol=tol, maxit=100)
    p = problems.SSR_FRANZ_DAM
    U, lh, oh, um, st = continuation.SSR_indirect_continuation(
        p["lambda_init"], p["d_lambda_init"], p["d_lambda_min"], p["d_lambda_diff_scaled_min"], p["step_max"],
        p["omega_max_stop"], p["it_newt_max"], p["it_damp_max"], p["tol"], p["r_min"], None, P.dmesh.mask,
        P.f_device(), P.cons, solver, max_steps_after_init=steps)
    return np.asarray(lh), np.asarray(oh), st


def test_franz_dam_seepage_and_ssr_match_oracle(cuda_device):
    g, P = _franz_problem(1e-10, 500)
    s = P.seepage
    assert s["stats"]["iterations"] == int(g["franz_newton"]) == int(g["stored_seepage_newton"])
    pw = s["pw"].cpu().numpy()
    assert np.max(np.abs(pw - g["franz_pw"])) <= 1e-8 * np.max(np.abs(g["franz_pw"]))
    assert np.array_equal(s["mater_sat"].cpu().numpy(), g["franz_sat"])
    lh, oh, st = _ssr(P, 1e-10, len(g["franz_its"]))
    assert np.max(np.abs(lh - g["franz_lambda"]) / g["franz_lambda"]) <= 1e-6
    assert np.max(np.abs(oh - g["franz_omega"]) / g["franz_omega"]) <= 1e-6
    assert list(st["step_newton_iterations"]) == list(g["franz_its"])


def test_franz_dam_reproduces_stored_run(cuda_device):
    g, P = _franz_problem(1e-6, 200)
    stored = g["stored_indirect_lambda"]
    lh, oh, st = _ssr(P, 1e-1, 4)
    assert abs(oh[0] - g["stored_indirect_omega_init"]) / g["stored_indirect_omega_init"] <= 1e-4
    assert np.max(np.abs(lh[2:] - stored[: len(lh) - 2]) / stored[: len(lh) - 2]) <= 1e-4


def test_scalar_amg_on_nonsymmetric_tangent(cuda_device):
    """The seepage tangent is not symmetric (its Bw' E C term): the scalar AMG takes the full
    Galerkin product, P'AP of the exported operators within 1e-12, and the coarse matrices
    keep the asymmetry."""
    from test_gpu_amg import export
    mesh, hat, dphi, W, n_q, Q_w, pw_D, conduct = _slope3d()
    dm = DeviceMesh(mesh, dphi, W, n_q)
    S = seepage.SeepageSystem(dm, hat, conduct, Q_w)
    eps = float(S.eps.max())
    pw = torch.from_numpy(np.where(pw_D > 0, pw_D, 0.5 * eps)).cuda()   # many points in the penalty band
    K, _ = S.system(pw, 2)
    amg = seepage.AMG(S.pattern)
    assert not amg.symmetric
    amg.update(K)
    nlev = len(amg.info()["levels"])
    assert nlev >= 2
    lev = export(amg, nlev)
    A0 = lev[0][0]
    assert abs(A0 - A0.T).max() > 1e-6 * abs(A0).max()
    for l in range(nlev - 1):
        A, Pd, _ = lev[l]
        Ac = (Pd.T @ A @ Pd).tocsr()
        Acd = lev[l + 1][0]
        dead = np.asarray(abs(Ac).sum(axis=1)).ravel() == 0
        Ac = Ac.tolil()
        for d in np.nonzero(dead)[0]:
            Ac[d, d] = 1.0
        assert abs(Acd - Ac.tocsr()).max() <= 1e-12 * abs(Ac).max()

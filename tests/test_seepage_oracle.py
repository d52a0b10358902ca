"""Seepage oracle and host set-up (CPU).

  * the oracle's restatement of SEEPAGE (oracle/seepage_ref.py) is pinned to the reference's
    stored run of slope_stability_2D_Franz_dam_SSR.ipynb: its seepage Newton converges in the
    stored 6 iterations on the Franz dam mesh, and the SSR indirect continuation on the
    seepage-coupled load (direct solves) gives omega_init and the lambda of the first three
    accepted steps within 1e-4 relative of the printed ones (the stored run used
    HYPRE-preconditioned DFGMRES at tolerance 1e-1 and Newton tolerance 1e-5);
  * the package's P1 -> P2 triangle conversion (fem.midpoints_p2_2d, vectorised) equals the
    oracle's element-by-element restatement of midpoints_P2.m bitwise, surf included;
  * the package's penalty parameters and boundary data equal the oracle's.
"""
import os

import numpy as np

from oracle import seepage_ref as sr
from slope_stability_octave_b200 import fem, problems, seepage

G = os.path.join(os.path.dirname(__file__), "golden", "seepage_oracle.npz")


def _franz():
    g = np.load(G)
    return g, sr.franz_dam_mesh(g["franz_coord_p1"], g["franz_elem_p1"], g["franz_mat"])


def test_oracle_pinned_to_stored_franz_dam_run():
    g = np.load(G)
    assert int(g["franz_newton"]) == int(g["stored_seepage_newton"]) == 6
    assert abs(g["franz_omega"][0] - g["stored_indirect_omega_init"]) / g["stored_indirect_omega_init"] <= 1e-4
    lam, stored = g["franz_lambda"][2:], g["stored_indirect_lambda"][: len(g["franz_lambda"]) - 2]
    assert np.max(np.abs(lam - stored) / stored) <= 1e-4


def test_oracle_seepage_reproduces_fixture():
    g, (coord, elem, Q, mater, surf) = _franz()
    mesh = fem.Mesh(coord, elem, Q)
    xi, wf = fem.quadrature_p2_tri()
    hat, d1, d2 = fem.local_basis_p2_tri(xi)
    D1, D2, W = fem.geometry_2d(mesh, d1, d2, wf)
    Q_w, pw_D = sr.franz_dam_seepage_bc(coord, surf)
    conduct = np.repeat(np.asarray(problems.FRANZ_DAM_K)[mater], wf.size)
    pw, _, sat, st = sr.seepage_problem(coord, elem, Q_w, pw_D, sr.GRHO, conduct, hat, (D1, D2), W)
    assert st["iterations"] == 6 and st["status"] == "converged"
    assert np.max(np.abs(pw - g["franz_pw"])) <= 1e-9 * np.max(np.abs(pw))
    assert np.array_equal(sat, g["franz_sat"])


def test_midpoints_p2_matches_restatement():
    g = np.load(G)
    c = g["franz_coord_p1"].T
    e = g["franz_elem_p1"].T
    a = sr.midpoints_p2_2d(c, e)
    b = fem.midpoints_p2_2d(c, e)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert a[0].shape[1] + c.shape[1] == 10049     # the stored run's node count


def test_penalty_and_boundary_data_match_oracle():
    g, (coord, elem, Q, mater, surf) = _franz()
    assert np.array_equal(seepage.penalty_parameters(coord, elem), sr.penalty_parameters(coord, elem))
    c2, e2, s2 = fem.mesh_p2_from_p1_2d(g["franz_coord_p1"].T, g["franz_elem_p1"].T)
    assert np.array_equal(c2, coord) and np.array_equal(e2, elem) and np.array_equal(s2, surf)
    for a, b in zip(problems.franz_dam_seepage_bc(coord, surf), sr.franz_dam_seepage_bc(coord, surf)):
        assert np.array_equal(a, b)
    assert int(Q.sum()) == 19848                  # the stored run's unknowns
    mesh = fem.mesh_p2_3d(1, 15, 10, 15, 10, 10, 1)
    assert np.array_equal(seepage.penalty_parameters(mesh.coord, mesh.elem),
                          sr.penalty_parameters(mesh.coord, mesh.elem))
    for a, b in zip(problems.homo_slope_seepage_bc(mesh.coord), sr.homo_slope_seepage_bc(mesh.coord)):
        assert np.array_equal(a, b)
    # the 3D penalty keeps the reference's L34 term: (x3-x4)^2 + (y3-y4)^2 + (z2-z4)^2
    X = np.array([[0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0], [0.0, 0.0, 0.0, 0.1]])
    eps = seepage.penalty_parameters(X, np.arange(4).reshape(4, 1))
    assert np.isclose(eps[0], sr.GRHO * 0.1 / 2)                    # L14 = 0.1
    X2 = np.array([[0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.9], [0.0, 0.0, 0.5, 0.1]])
    eps2 = seepage.penalty_parameters(X2, np.arange(4).reshape(4, 1))
    # the true L34 would be sqrt(0.1^2 + 0.4^2); the reference's term gives sqrt(0.1^2 + 0.1^2)
    assert np.isclose(eps2[0], sr.GRHO * np.sqrt(0.1 ** 2 + 0.1 ** 2) / 2)

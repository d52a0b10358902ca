"""Pin the oracle: its C restatement must reproduce the reference's own C kernels.

Against the golden fixtures (generated from the reference MEX sources, always available)
and, when oracle/_ref is built from the reference tree, against the live reference.
"""
import os

import numpy as np
import pytest

from oracle import native
from oracle.octave_ref import OctavePattern, assemble_via_oracle
from slope_stability_octave_b200 import fem, workloads

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def test_golden_constitutive_3d_bitwise():
    g = _load("constitutive_3d.npz")
    S, DS, br = native.constitutive(3, g["E"], g["c_bar"], g["sin_phi"], g["shear"], g["bulk"], g["lame"])
    assert np.array_equal(br, g["branch"])
    assert np.array_equal(S, g["S"])
    assert np.array_equal(DS, g["DS"])
    assert np.all(np.bincount(br, minlength=5) == 200)


def test_golden_constitutive_2d_bitwise():
    g = _load("constitutive_2d.npz")
    S, DS, br = native.constitutive(2, g["E"], g["c_bar"], g["sin_phi"], g["shear"], g["bulk"], g["lame"])
    assert np.array_equal(S, g["S"])
    assert np.array_equal(DS, g["DS"])
    counts = np.bincount(br, minlength=5)
    assert counts[0] > 0 and counts[1] > 0 and counts[4] > 0


def _small3d():
    m = fem.mesh_p2_3d(1, 2, 1, 2, 1, 1, 2)
    xi, wf = fem.quadrature_p2_tet()
    _, a, b, c = fem.local_basis_p2_tet(xi)
    d1, d2, d3, w = fem.geometry_3d(m, a, b, c, wf)
    mat = fem.materials(np.zeros(m.n_e, int), 11, [6, 45, 0, 40000, 0.3, 20, 20])
    return m, (d1, d2, d3), w, mat


def test_golden_pattern_and_assembly_3d():
    g = _load("assembly_3d.npz")
    m, dphi, w, mat = _small3d()
    pat = OctavePattern(3, m.elem, m.n_n, dphi, w, m.Q, mat["shear"], mat["bulk"])
    assert np.array_equal(pat.ref_I, g["ref_I"]) and np.array_equal(pat.ref_J, g["ref_J"])
    assert np.array_equal(pat.transpose_perm, g["transpose_perm"])
    np.testing.assert_allclose(pat.V_elast, g["V_elast"], rtol=1e-13, atol=1e-9)
    V, smap = assemble_via_oracle(pat, dphi, g["DS"], 11)
    assert np.array_equal(smap, g["scatter_map"])
    assert np.array_equal(V, g["V_tang"])


def test_golden_pattern_and_assembly_2d():
    g = _load("assembly_2d.npz")
    m = fem.mesh_p2_2d(1.0, 3, 2, 3, 2, 2)
    xi, wf = fem.quadrature_p2_tri()
    _, a, b = fem.local_basis_p2_tri(xi)
    d1, d2, w = fem.geometry_2d(m, a, b, wf)
    mat = fem.materials(np.zeros(m.n_e, int), 7, [6, 45, 0, 40000, 0.3, 20, 20])
    pat = OctavePattern(2, m.elem, m.n_n, (d1, d2), w, m.Q, mat["shear"], mat["bulk"])
    assert np.array_equal(pat.ref_I, g["ref_I"]) and np.array_equal(pat.ref_J, g["ref_J"])
    np.testing.assert_allclose(pat.V_elast, g["V_elast"], rtol=1e-13, atol=1e-9)
    V, smap = assemble_via_oracle(pat, (d1, d2), g["DS"], 7)
    assert np.array_equal(smap, g["scatter_map"])
    assert np.array_equal(V, g["V_tang"])


def test_pattern_equals_node_adjacency_on_free_dofs():
    """The maximal symbolic pattern of K(Q,Q) is the node adjacency (x) 3x3 restricted to Q."""
    import scipy.sparse as sp
    m, dphi, w, mat = _small3d()
    pat = OctavePattern(3, m.elem, m.n_n, dphi, w, m.Q, mat["shear"], mat["bulk"])
    r = np.repeat(m.elem.T, 10, axis=1).ravel()
    c = np.tile(m.elem.T, (1, 10)).ravel()
    A = sp.coo_matrix((np.ones(r.size), (r, c)), shape=(m.n_n, m.n_n)).tocsr()
    A.data[:] = 1
    Ad = sp.kron(A, np.ones((3, 3))).tocsc()[pat.Q_flat][:, pat.Q_flat].tocsc()
    Ad.sort_indices()
    J = np.repeat(np.arange(pat.n_Q), np.diff(Ad.indptr))
    assert np.array_equal(Ad.indices + 1, pat.ref_I) and np.array_equal(J + 1, pat.ref_J)


def test_assembly_matches_global_spmm():
    """Element assembly equals the reference's global B_Q' D B_Q path (CONSTITUTIVE.m:503-513)."""
    m, dphi, w, mat = _small3d()
    pat = OctavePattern(3, m.elem, m.n_n, dphi, w, m.Q, mat["shear"], mat["bulk"])
    d = workloads.constitutive_points(w.size, seed=3)
    _, DS, _ = native.constitutive(3, d["E"], d["c_bar"], d["sin_phi"], mat["shear"], mat["bulk"], mat["lame"])
    V, _ = assemble_via_oracle(pat, dphi, DS, 11)
    Vg = pat.assemble_tangent_global(DS)
    assert np.max(np.abs(V - Vg)) <= 1e-13 * np.max(np.abs(Vg))


@pytest.mark.skipif(not native.ref_available(), reason="reference build (oracle/_ref) not present")
def test_live_reference_constitutive_bitwise():
    for seed in (1, 2):
        d = workloads.constitutive_points(20000, seed=seed)
        for want in (True, False):
            S, DS, _ = native.constitutive(3, d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"], want)
            Sr, DSr = native.ref_constitutive(3, d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"], want)
            assert np.array_equal(S, Sr)
            if want:
                assert np.array_equal(DS, DSr)
    rng = np.random.default_rng(4)
    n = 20000
    E = rng.normal(size=(n, 3)) * 1e-3
    cb, sp = native.reduction(rng.uniform(5, 15, n), np.deg2rad(rng.uniform(25, 45, n)), np.zeros(n), 1.2)
    G, K = np.full(n, 40000 / 2.6), np.full(n, 40000 / 1.2)
    L = K - 2 * G / 3
    S, DS, _ = native.constitutive(2, E, cb, sp, G, K, L)
    Sr, DSr = native.ref_constitutive(2, E, cb, sp, G, K, L)
    assert np.array_equal(S, Sr) and np.array_equal(DS, DSr)


def test_reduction_matches_host_restatement():
    rng = np.random.default_rng(5)
    n = 1000
    c0 = rng.uniform(5, 15, n)
    phi = np.deg2rad(rng.uniform(25, 45, n))
    psi = np.deg2rad(rng.uniform(0, 10, n))
    for davis in "AB":
        for lam in (0.7, 1.0, 1.6):
            cb, sp = native.reduction(c0, phi, psi, lam, davis)
            cb2, sp2 = fem.davis_reduction(c0, phi, psi, lam, davis)
            np.testing.assert_allclose(cb, cb2, rtol=1e-14)
            np.testing.assert_allclose(sp, sp2, rtol=1e-14)


def test_oracle_continuation_reproduces_fixture():
    """The oracle's 2D SSR continuation (direct solver) reproduces ssr_oracle.npz."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_continuation_golden import cases, run_case
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ssr_oracle.npz"))
    make, params = cases()["slope2d"]
    lh, oh, its = run_case(make, params)
    np.testing.assert_allclose(lh, g["slope2d_lambda"], rtol=1e-10)
    np.testing.assert_allclose(oh, g["slope2d_omega"], rtol=1e-10)
    assert list(its) == list(g["slope2d_newton"])


def test_oracle_layered_and_random_field_fixtures_reproduce():
    """The heterogeneous-material fixtures regenerate exactly from their script: the layered
    slope's SSR history (per-element materials) and the random-field slope's LL history
    (per-point lognormal c and phi from the seeded circulant-embedding field)."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_continuation_golden import layered_cases, ll_cases, run_case, run_ll_case
    gdir = os.path.join(os.path.dirname(__file__), "golden")
    g = np.load(os.path.join(gdir, "ssr_oracle.npz"))
    make, params = layered_cases()["layered3d"]
    lh, oh, its = run_case(make, params)
    np.testing.assert_allclose(lh, g["layered3d_lambda"], rtol=1e-10)
    np.testing.assert_allclose(oh, g["layered3d_omega"], rtol=1e-10)
    assert list(its) == list(g["layered3d_newton"])
    g = np.load(os.path.join(gdir, "ll_oracle.npz"))
    make, p = ll_cases()["rf3d"]
    th, oh, its = run_ll_case(make, p)
    np.testing.assert_allclose(th, g["rf3d_t"], rtol=1e-10)
    np.testing.assert_allclose(oh, g["rf3d_omega"], rtol=1e-10)
    assert list(its) == list(g["rf3d_newton"])

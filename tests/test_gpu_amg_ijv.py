"""The id-keyed preconditioner instances over host COO triplets (the hypre_boomeramg_mex
command set: setup_ijv / update_values / apply / clear, hypre_boomeramg_mex.cpp:751-1270)
through the C ABI, on the oracle's K_r(Q,Q) of a small 3D slope.

The caller's side is the reference's: I, J, V of the full matrix as 1-based doubles in the
order of Octave's find, the near-null space of near_null_space_elasticity_3D.m (rigid-body
modes on the free DOFs, orthonormalised), dof_func = mod(q - 1, 3) as set_linear_solver.m
builds it.  The oracle's DFGMRES (dfgmres_solver.m restated) preconditioned by
sg_amg_apply_host must reach 1e-8 within the iteration count of the device path's own AMG on
the same matrix plus a small margin; a value update keeps the pattern; a repeated
setup_ijv with the same triplet count takes the value-only path; clear forgets the id.
"""
import ctypes as C

import numpy as np
import pytest

from slope_stability_octave_b200 import _lib, problems
from slope_stability_octave_b200.linear_solvers import near_null_space_elasticity

pytestmark = pytest.mark.gpu

ID = b"test_ijv_instance"


def hp(a):
    return a.ctypes.data_as(C.c_void_p)


def reference_side(P, cons, U, lam, r):
    """(I, J, V, n, Z, dof_func) as the reference's newton_ind_SSR.m passes them."""
    from oracle.drivers import OracleConstitutive  # noqa: F401  (type of cons)
    cons.reduction(lam)
    cons.build_F_and_DS_reduced(U)
    K = cons.build_K_r_QQ_vals(r).tocsc()
    K.sort_indices()
    n = K.shape[0]
    J = np.repeat(np.arange(n), np.diff(K.indptr)).astype(np.float64) + 1
    I = K.indices.astype(np.float64) + 1
    V = K.data.astype(np.float64).copy()
    Qf = P.mesh.Q.T.ravel()
    q = np.nonzero(Qf)[0]
    Zr = near_null_space_elasticity(P.mesh.coord, P.mesh.Q)[q]
    Z, _ = np.linalg.qr(Zr)                     # orthonormal columns, as the reference's MGS
    dof_func = (q % 3).astype(np.float64)       # mod(q_idx - 1, 3) with 1-based q_idx
    return K, I, J, V, n, np.asfortranarray(Z), dof_func


def setup(I, J, V, n, Z, dof_func, force=0):
    t = C.c_double()
    rc = _lib.lib().sg_amg_setup_ijv(ID, hp(I), hp(J), hp(V), V.size, n, hp(Z), Z.shape[1], hp(dof_func), 3,
                                     None, 0, force, C.byref(t))
    assert rc == 0, _lib.lib().sg_last_error()
    return t.value


def info():
    buf = np.zeros(8, np.int64)
    assert _lib.lib().sg_amg_ijv_info(ID, hp(buf), 8) == 0
    return dict(zip(["n", "nnz", "b", "nns", "nodes", "blocks", "full_builds", "value_updates"], buf.tolist()))


def apply(n):
    def M(r):
        r = np.ascontiguousarray(r, np.float64)
        y = np.empty(n)
        rc = _lib.lib().sg_amg_apply_host(ID, hp(r), hp(y), n)
        assert rc == 0, _lib.lib().sg_last_error()
        return y
    return M


def device_iterations(P, lam, r, tol):
    """FGMRES iterations of the device path (mesh block pattern, its own AMG) on the K_r of
    the elastic state at (lam, r), the matrix the oracle assembles for U = 0."""
    import torch
    P.to_device()
    P.cons.init_K_r_pattern()
    P.cons.reduction(lam)
    P.cons.build_F_and_DS_reduced(torch.zeros(P.dmesh.n_dof, dtype=torch.float64, device="cuda"))
    Kd = P.cons.build_K_r_QQ_vals(r)
    solver = P.solver("DFGMRES_B200", tol=tol, maxit=200)
    solver.setup_preconditioner(Kd)
    b = P.f_device() * P.dmesh.mask
    _, its = solver.solve(Kd, b)
    return its


def test_ijv_instance_preconditions_dfgmres(cuda_device):
    from oracle.drivers import OracleConstitutive, dfgmres
    _lib.lib().sg_amg_clear(None)
    P = problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 2))
    cons = OracleConstitutive(P.mesh, P.dphi, P.weight, P.n_q, P.mat)
    n_full = P.mesh.Q.size
    U0 = np.zeros(n_full)
    K, I, J, V, n, Z, dof_func = reference_side(P, cons, U0, 1.0, 1e-4)
    t_full = setup(I, J, V, n, Z, dof_func)
    d = info()
    assert d["n"] == n and d["nnz"] == V.size and d["b"] == 3 and d["nns"] == 6 and d["full_builds"] == 1
    # every node of the mesh with a free DOF is one block row
    assert d["nodes"] == int(P.mesh.Q.any(axis=0).sum())
    Qf = P.mesh.Q.T.ravel()
    f = np.ascontiguousarray(P.f.T).ravel()[Qf]
    x, its, hist = dfgmres(K, f, apply(n), None, 200, 1e-8)
    assert hist[-1] < 1e-8
    assert np.linalg.norm(f - K @ x) <= 1.1e-8 * np.linalg.norm(f)
    # about the iterations of the device path's own AMG on the same matrix
    assert its <= device_iterations(P, 1.0, 1e-4, 1e-8) + 5
    # plastic values on the same pattern: value update, same instance
    Qm = np.zeros(n_full, bool)
    Qm[np.nonzero(Qf)[0]] = True
    Ue = np.zeros(n_full)
    Ue[Qm] = 4.0 * x
    K2, I2, J2, V2, _, _, _ = reference_side(P, cons, Ue, 1.4, 1e-2)
    assert np.array_equal(I2, I) and np.array_equal(J2, J)
    t = C.c_double()
    rc = _lib.lib().sg_amg_update_values(ID, hp(V2), V2.size, C.byref(t))
    assert rc == 0, _lib.lib().sg_last_error()
    assert info()["value_updates"] == 1 and info()["full_builds"] == 1
    x2, its2, hist2 = dfgmres(K2, f, apply(n), None, 200, 1e-8)
    assert hist2[-1] < 1e-8
    assert np.linalg.norm(f - K2 @ x2) <= 1.1e-8 * np.linalg.norm(f)
    # setup_ijv again with the same triplet count: the value-only path (the reference's
    # pattern reuse), faster than the first build
    t_fast = setup(I2, J2, V2, n, Z, dof_func)
    assert info()["full_builds"] == 1 and info()["value_updates"] == 2
    assert t_fast < t_full
    r = np.random.default_rng(0).normal(size=n)
    # force_rebuild: a new instance
    setup(I2, J2, V2, n, Z, dof_func, force=1)
    assert info()["full_builds"] == 1 and info()["value_updates"] == 0
    assert _lib.lib().sg_amg_clear(ID) == 0
    buf = np.zeros(8, np.int64)
    assert _lib.lib().sg_amg_ijv_info(ID, hp(buf), 8) == -4
    y = np.empty(n)
    assert _lib.lib().sg_amg_apply_host(ID, hp(r), hp(y), n) == -4


def test_ijv_instance_without_near_null_space_and_duplicates(cuda_device):
    """No Z (translations only), no dof_func (q mod 3), and every triplet given twice with half
    its value (duplicates are summed): the same preconditioner as the plain triplets."""
    from oracle.drivers import OracleConstitutive, dfgmres
    _lib.lib().sg_amg_clear(None)
    P = problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 1))
    cons = OracleConstitutive(P.mesh, P.dphi, P.weight, P.n_q, P.mat)
    K, I, J, V, n, Z, dof_func = reference_side(P, cons, np.zeros(P.mesh.Q.size), 1.0, 1e-4)
    L = _lib.lib()
    rc = L.sg_amg_setup_ijv(ID, hp(I), hp(J), hp(V), V.size, n, None, 0, None, 3, None, 0, 0, None)
    assert rc == 0, L.sg_last_error()
    r = np.random.default_rng(1).normal(size=n)
    y1 = apply(n)(r)
    I2 = np.concatenate([I, I])
    J2 = np.concatenate([J, J])
    V2 = np.concatenate([V / 2, V / 2])
    rc = L.sg_amg_setup_ijv(b"dup", hp(I2), hp(J2), hp(V2), V2.size, n, None, 0, None, 3, None, 0, 0, None)
    assert rc == 0, L.sg_last_error()
    y2 = np.empty(n)
    assert L.sg_amg_apply_host(b"dup", hp(r), hp(y2), n) == 0
    assert np.allclose(y1, y2, rtol=1e-10, atol=1e-12 * np.abs(y1).max())
    Qf = P.mesh.Q.T.ravel()
    f = np.ascontiguousarray(P.f.T).ravel()[Qf]
    _, its, hist = dfgmres(K, f, apply(n), None, 200, 1e-8)
    assert hist[-1] < 1e-8
    buf = np.zeros(1, np.int64)
    assert L.sg_amg_ijv_info(None, hp(buf), 1) == 0 and buf[0] == 2
    assert L.sg_amg_clear(None) == 0
    assert L.sg_amg_ijv_info(None, hp(buf), 1) == 0 and buf[0] == 0

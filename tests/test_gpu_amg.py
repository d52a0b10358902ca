"""GPU parity of the AMG preconditioner against the oracle's SciPy restatement of the same
algorithm (oracle/amg_ref.py).  BoomerAMG itself is not available, so parity is with the
algorithm this build implements.

  * hierarchy sizes (aggregation on the strength graph) equal the restatement's;
  * device prolongators equal T - omega D^-1 A T from the restatement within 1e-10 relative
    (omega comes from a 10-step power iteration on both sides);
  * each coarse matrix equals P' A P of the exported level within 1e-12 relative;
  * one V-cycle equals the restatement's V-cycle on the exported hierarchy within 1e-10;
  * the mixed-precision (FP32) cycle agrees with the FP64 cycle to FP32 accuracy (1e-4).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle.amg_ref import Hierarchy
from slope_stability_octave_b200 import _lib, problems
from slope_stability_octave_b200.device import hptr, ptr
from slope_stability_octave_b200.linear_solvers import AMG, near_null_space_elasticity

pytestmark = pytest.mark.gpu


def export(amg, nlev):
    info = amg.info()
    out = []
    for l in range(nlev):
        L = info["levels"][l]
        b, n, nb = L["block"], L["rows"], L["blocks"]
        rp = np.zeros(n + 1, np.int32)
        col = np.zeros(nb, np.int32)
        vals = np.zeros(nb * b * b)
        P = None
        if l + 1 < nlev:
            bc, nc = info["levels"][l + 1]["block"], info["levels"][l + 1]["rows"]
            prp = np.zeros(n + 1, np.int32)
            _lib.call("sg_amg_export", amg.handle, l, None, None, None, hptr(prp), None, None)
            pnb = int(prp[-1])
            pcol = np.zeros(pnb, np.int32)
            pv = np.zeros(pnb * b * bc)
            _lib.call("sg_amg_export", amg.handle, l, hptr(rp), hptr(col), hptr(vals), hptr(prp), hptr(pcol), hptr(pv))
            P = sp.bsr_matrix((pv.reshape(-1, b, bc), pcol, prp), shape=(n * b, nc * bc)).tocsr()
        else:
            _lib.call("sg_amg_export", amg.handle, l, hptr(rp), hptr(col), hptr(vals), None, None, None)
        A = sp.bsr_matrix((vals.reshape(-1, b, b), col, rp), shape=(n * b, n * b)).tocsr()
        out.append((A, P, b))
    return out


def elastic_problem():
    P = problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 2)).to_device()
    P.cons.init_K_r_pattern()
    f = P.f_device()
    P.cons.reduction(1.0)
    P.cons.build_F_and_DS_reduced(torch.zeros_like(f))
    K = P.cons.build_K_r_QQ_vals(1e-4)
    return P, K


@pytest.mark.parametrize("theta", [0.02, 0.0])
def test_amg_hierarchy_and_vcycle_match_restatement(cuda_device, theta):
    P, K = elastic_problem()
    amg = AMG(P.dmesh, theta=theta)
    amg.update(K)
    info = amg.info()
    nlev = len(info["levels"])
    assert nlev >= 2
    lev = export(amg, nlev)
    Kh = lev[0][0]
    Qm = P.mesh.Q.T.ravel()
    B = near_null_space_elasticity(P.mesh.coord, P.mesh.Q)
    H = Hierarchy(Kh, B, 3, fixed=~Qm, theta=theta)
    assert [l["A"].shape[0] for l in H.levels] == [A.shape[0] for A, _, _ in lev]
    for l in range(nlev - 1):
        A, Pd, b = lev[l]
        Ph = H.levels[l]["P"]
        assert abs(Pd - Ph).max() <= 1e-10 * abs(Ph).max()
        Ac = (Pd.T @ A @ Pd).tocsr()
        Acd = lev[l + 1][0]
        dead = H.levels[l + 1].get("dead")
        if dead is not None and dead.any():
            Ac = Ac.tolil()
            for d in np.nonzero(dead)[0]:
                Ac[d, :] = 0
                Ac[:, d] = 0
                Ac[d, d] = 1.0
            Ac = Ac.tocsr()
        assert abs(Acd - Ac).max() <= 1e-12 * abs(Ac).max()
    # V-cycle on the exported hierarchy
    Hx = Hierarchy.from_levels([A for A, _, _ in lev], [p for _, p, _ in lev[:-1]], [b for _, _, b in lev])
    rng = np.random.default_rng(0)
    r = rng.normal(size=Kh.shape[0]) * Qm
    rd = torch.from_numpy(r).to(cuda_device)
    zd = torch.zeros_like(rd)
    amg.apply(rd, zd)
    torch.cuda.synchronize()
    z = zd.cpu().numpy()
    zr = Hx.vcycle(r)
    assert np.linalg.norm(z - zr) <= 1e-10 * np.linalg.norm(zr)


def test_amg_mixed_precision_cycle(cuda_device):
    P, K = elastic_problem()
    a64 = AMG(P.dmesh)
    a32 = AMG(P.dmesh, mixed=True, fine_half=False)
    a64.update(K)
    a32.update(K)
    rng = np.random.default_rng(1)
    r = torch.from_numpy(rng.normal(size=P.dmesh.n_dof) * P.mesh.Q.T.ravel()).to(cuda_device)
    z64, z32 = torch.zeros_like(r), torch.zeros_like(r)
    a64.apply(r, z64)
    a32.apply(r, z32)
    torch.cuda.synchronize()
    err = torch.linalg.norm(z64 - z32) / torch.linalg.norm(z64)
    assert err.item() < 1e-4


def test_amg_mixed_cycle_with_fp16_level0(cuda_device):
    # the FP32 cycle whose level-0 SpMVs read the FP16 copy of A (11-bit significand, values
    # scaled by a power of two): the cycle agrees with the FP64 one to FP16 accuracy (1e-2),
    # and DFGMRES preconditioned by it reaches the same FP64 residual tolerance
    from slope_stability_octave_b200.linear_solvers import DFGMRES
    P, K = elastic_problem()
    a64 = AMG(P.dmesh)
    a16 = AMG(P.dmesh, mixed=True, fine_half=True)
    a64.update(K)
    a16.update(K)
    rng = np.random.default_rng(1)
    r = torch.from_numpy(rng.normal(size=P.dmesh.n_dof) * P.mesh.Q.T.ravel()).to(cuda_device)
    z64, z16 = torch.zeros_like(r), torch.zeros_like(r)
    a64.apply(r, z64)
    a16.apply(r, z16)
    torch.cuda.synchronize()
    err = torch.linalg.norm(z64 - z16) / torch.linalg.norm(z64)
    assert 0 < err.item() < 1e-2
    its = []
    for amg in (a64, a16):
        s = DFGMRES(P.dmesh, 1e-8, 200, 1e-3, amg=amg)
        x, it = s.solve(K, r)
        res = torch.zeros_like(r)
        P.dmesh.spmv(K, x, res)
        assert torch.linalg.norm((r - res) * P.dmesh.mask).item() <= 1e-7 * torch.linalg.norm(r).item()
        its.append(it)
    assert its[1] <= its[0] + 2


def test_amg_apply_before_update_is_an_error(cuda_device):
    P, K = elastic_problem()
    amg = AMG(P.dmesh)
    amg.update(K)
    # a second hierarchy that never received values refuses to apply
    h = C.c_void_p()
    Z = np.ascontiguousarray(near_null_space_elasticity(P.mesh.coord, P.mesh.Q).T)
    _lib.call("sg_amg_create", P.dmesh.bsr, None, hptr(Z), 6, None, None, 0, C.byref(h), None)
    r = torch.zeros(P.dmesh.n_dof, dtype=torch.float64, device=cuda_device)
    rc = _lib.lib().sg_amg_apply(h, ptr(r), ptr(r), None)
    assert rc == -4
    _lib.lib().sg_amg_destroy(h)


def test_symmetric_galerkin_mirror(cuda_device):
    """K_r is symmetric, so the AMG forms each coarse matrix on and above its block diagonal
    and mirrors it (option symmetric): the blocks off the diagonal of every coarse level are
    exact transposes of each other, and the matrices agree with the full product (option off)
    to rounding."""
    P, K = elastic_problem()
    a_sym = AMG(P.dmesh)
    a_full = AMG(P.dmesh, symmetric=False)
    assert a_sym.symmetric and not a_full.symmetric
    a_sym.update(K)
    a_full.update(K)
    nlev = len(a_sym.info()["levels"])
    ls, lf = export(a_sym, nlev), export(a_full, nlev)
    for l in range(1, nlev):
        As, Af = ls[l][0], lf[l][0]
        b = ls[l][2]
        D = (As - As.T).tocoo()
        off = (D.row // b) != (D.col // b)
        # blocks off the diagonal are mirrored copies; inside a diagonal block the two
        # triangles are separate sums and agree to rounding
        assert np.all(D.data[off] == 0.0)
        assert abs(D.data).max(initial=0.0) <= 1e-14 * abs(As).max()
        assert abs(As - Af).max() <= 1e-12 * abs(Af).max()

"""The learned node-wise V-cycle correction on the GPU against its CPU oracle
(oracle/learned_ref.py), and what the trained network gains.

  * tensor-core forward pass (sg_mlp_forward_dev) against the oracle with the same BF16
    rounding points: output within 1e-2 of its scale (FP32 accumulation order and rare
    one-ulp BF16 differences of hidden activations are the only differences);
  * tensor-core backward pass (sg_mlp_backward_dev): every parameter group's gradient within
    3e-2 relative (norm) of the oracle's;
  * node features of a plastic Newton system of the 3D slope within one BF16 ulp of the
    oracle's; the diagonal-block inverses within 1e-12;
  * the training loss and its parameter gradient through the whole chain (network, 3x3
    correction, FP64 SpMVs, backward) against the oracle on the vectors the GPU collected:
    loss within 1e-6, gradient within 3e-2 relative per group, for both objectives;
  * the gain: after training on residual vectors of the Newton system's own right-hand side,
    the corrected V-cycle leaves a smaller residual on held-out vectors of another right-hand
    side than the plain V-cycle (objective < 0.9, the plain cycle's is exactly 1), and DFGMRES
    at the continuation's linear tolerance (1e-1) needs no more iterations with it than
    without (at 1e-6 at most 4 more: the local correction is not symmetric);
  * the DFGMRES hook trains at its first solve, runs the acceptance trial (plain vs
    corrected solve of the training system; the correction is kept only if it needs fewer
    iterations) and returns a solution at the tolerance.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import learned_ref as LR
from slope_stability_octave_b200 import _lib, continuation, problems
from slope_stability_octave_b200.device import ptr
from slope_stability_octave_b200.learned import LearnedCorrection
from slope_stability_octave_b200.linear_solvers import AMG, DFGMRES, set_linear_solver

pytestmark = pytest.mark.gpu

GROUPS = [("W1", LR.OFF_W1, LR.OFF_B1), ("b1", LR.OFF_B1, LR.OFF_W2), ("W2", LR.OFF_W2, LR.OFF_B2),
          ("b2", LR.OFF_B2, LR.OFF_W3), ("W3", LR.OFF_W3, LR.OFF_B3), ("b3", LR.OFF_B3, LR.NPARAM)]


def group_errors(g, ref):
    return {name: float(np.linalg.norm(g[a:b] - ref[a:b]) / max(np.linalg.norm(ref[a:b]), 1e-30))
            for name, a, b in GROUPS}


def random_features(n, seed):
    rng = np.random.default_rng(seed)
    n_pad = (n + 127) // 128 * 128
    X = np.zeros((n_pad, 16), np.float32)
    X[:n] = rng.uniform(-2, 2, (n, 16))
    return LR.bf16(X), n_pad


def test_forward_matches_oracle(cuda_device):
    n = 1000
    X, n_pad = random_features(n, 1)
    p = LR.init_params(5, zero_last=False)
    Xd = torch.from_numpy(LR.bf16_bits(X).view(np.int16)).to(cuda_device)
    pd = torch.from_numpy(p).to(cuda_device)
    G = torch.zeros((n_pad, 16), dtype=torch.float32, device=cuda_device)
    err = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    _lib.call("sg_mlp_forward_dev", ptr(pd), ptr(Xd), n, ptr(G), ptr(err), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    Y, _ = LR.mlp_forward(p, X[:n])
    Gh = G.cpu().numpy()[:n]
    scale = np.abs(Y).max()
    assert np.abs(Gh - Y).max() <= 1e-2 * scale
    assert np.linalg.norm(Gh - Y) <= 2e-3 * np.linalg.norm(Y)
    assert np.all(G.cpu().numpy()[n:] == 0)


def test_backward_matches_oracle(cuda_device):
    n = 1000
    X, n_pad = random_features(n, 2)
    p = LR.init_params(6, zero_last=False)
    rng = np.random.default_rng(3)
    dG = np.zeros((n_pad, 16), np.float32)
    dG[:n] = rng.normal(size=(n, 16))
    Xd = torch.from_numpy(LR.bf16_bits(X).view(np.int16)).to(cuda_device)
    pd = torch.from_numpy(p).to(cuda_device)
    dGd = torch.from_numpy(dG).to(cuda_device)
    grad = torch.zeros(LR.NPARAM, dtype=torch.float32, device=cuda_device)
    part = torch.zeros(int(_lib.lib().sg_mlp_part_size(n)), dtype=torch.float32, device=cuda_device)
    err = torch.zeros(1, dtype=torch.int32, device=cuda_device)
    _lib.call("sg_mlp_backward_dev", ptr(pd), ptr(Xd), ptr(dGd), n, ptr(grad), ptr(part), ptr(err),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = LR.mlp_backward(p, X, dG)
    errs = group_errors(grad.cpu().numpy().astype(np.float64), ref)
    assert max(errs.values()) <= 3e-2, errs


@pytest.fixture(scope="module")
def system(cuda_device):
    """A plastic Newton system of the 3D slope (z = 2 m): two accepted SSR steps after the
    init phase, then the tangent K_r and the equilibrium residual at the last lambda."""
    P = problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 2)).to_device()
    solver = P.solver("DFGMRES_B200", tol=1e-1, maxit=100)
    p = problems.SSR_3D
    f = P.f_device()
    U, lh, oh, um, st = continuation.SSR_indirect_continuation(
        p["lambda_init"], p["d_lambda_init"], p["d_lambda_min"], p["d_lambda_diff_scaled_min"], p["step_max"],
        p["omega_max_stop"], p["it_newt_max"], p["it_damp_max"], p["tol"], p["r_min"], None, P.dmesh.mask, f,
        P.cons, solver, max_steps_after_init=2)
    lam = float(lh[-1])
    F = P.cons.build_F_and_DS_all(lam, U)
    K = P.cons.build_K_r_QQ_vals(1e-4).clone()
    b = (f - F) * P.dmesh.mask
    amg = AMG(P.dmesh, mixed=False)
    amg.update(K)
    I, J, _ = P.dmesh.pattern()
    V = P.dmesh.to_ref(K).cpu().numpy()
    q = P.dmesh.free_dofs()
    n = P.dmesh.n_dof
    KQ = sp.csr_matrix((V, (I - 1, J - 1)), shape=(q.size, q.size))
    E = sp.csr_matrix((np.ones(q.size), (q, np.arange(q.size))), shape=(n, q.size))
    fixed = np.ones(n)
    fixed[q] = 0.0
    A = (E @ KQ @ E.T + sp.diags(fixed)).tocsr()
    torch.cuda.synchronize()
    return dict(P=P, K=K, b=b, f=f, amg=amg, A=A, lam=lam, branch_mix=np.bincount(
        P.cons.branch.cpu().numpy(), minlength=5))


def oracle_inputs(s):
    P, A = s["P"], s["A"]
    nn = P.dmesh.n_n
    d0 = A.diagonal()
    # 3x3 diagonal blocks from the CSR rows (vectorised)
    Kd = np.zeros((nn, 3, 3))
    Ac = A.tocoo()
    sel = (Ac.row // 3) == (Ac.col // 3)
    Kd[Ac.row[sel] // 3, Ac.row[sel] % 3, Ac.col[sel] % 3] = Ac.data[sel]
    assert np.allclose(Kd[:, [0, 1, 2], [0, 1, 2]].ravel(), d0)
    mask = P.dmesh.mask.cpu().numpy().reshape(nn, 3)
    return Kd, mask


def test_features_and_block_inverse_match_oracle(system):
    s = system
    P = s["P"]
    assert s["branch_mix"][1:].sum() > 0, "the system must have plastic points"
    lc = LearnedCorrection(P.dmesh, cons=P.cons)
    lc.features(s["K"], s["b"])
    Kd, mask = oracle_inputs(s)
    nn = P.dmesh.n_n
    ref = LR.bf16(LR.features(Kd, mask, P.mesh.coord, s["b"].cpu().numpy().reshape(nn, 3), P.mesh.elem, P.n_q,
                              P.cons.branch.cpu().numpy(), P.cons.c_bar.cpu().numpy()))
    got = lc.export("features")
    assert np.all(got[nn:] == 0)
    diff = np.abs(got[:nn] - ref)
    assert np.all(diff <= 2.0 ** -7 * np.maximum(np.abs(ref), 1e-3)), float(diff.max())
    Dinv = lc.export("Dinv")
    Dref = LR.block_inv(Kd)
    assert np.abs(Dinv - Dref).max() <= 1e-12 * np.abs(Dref).max()


def test_training_gradient_matches_oracle(system):
    s = system
    P = s["P"]
    nn = P.dmesh.n_n
    lc = LearnedCorrection(P.dmesh, cons=P.cons, max_vectors=6)
    lc.features(s["K"], s["b"])
    lc.collect(s["amg"], s["K"], s["b"], 6, slot=0)
    p = LR.init_params(11, zero_last=False)
    p[LR.OFF_W3:LR.OFF_B3] *= 0.05
    lc.set_params(p)
    X = lc.export("features")
    Dinv = lc.export("Dinv")
    rz = [lc.export("rz0", i) for i in range(6)]
    _, mask = oracle_inputs(s)
    Y, _ = LR.mlp_forward(p, X)
    for kind, code in (("energy", 1), ("residual", 0)):
        _lib.call("sg_learned_set_loss", lc.handle, code)
        g, loss = lc.gradient(s["K"], slot=0)
        loss_ref, dG = LR.correction_loss(Y[:nn], Dinv, mask, s["A"], rz, kind)
        assert abs(loss - loss_ref) <= 1e-6 * abs(loss_ref), kind
        dGp = np.zeros((X.shape[0], 16))
        dGp[:nn] = dG
        ref = LR.mlp_backward(p, X, dGp.astype(np.float32))
        errs = group_errors(g.astype(np.float64), ref)
        assert max(errs.values()) <= 3e-2, (kind, errs)


def test_trained_correction_gains_over_plain_vcycle(system):
    s = system
    P, K, amg = s["P"], s["K"], s["amg"]
    lc = LearnedCorrection(P.dmesh, cons=P.cons, n_vectors=12, steps=80, lr=3e-3, seed=1, max_vectors=12)
    lc.features(K, s["b"])
    lc.collect(amg, K, s["b"], 12, slot=0)
    lc.collect(amg, K, s["f"] * P.dmesh.mask, 4, slot=1)
    assert lc.loss(K, slot=1) == pytest.approx(1.0, abs=1e-12)     # untrained: the plain cycle
    hist = lc.train(K)
    held = lc.loss(K, slot=1)
    print(f"residual objective: train {hist[0]:.4f} -> {hist[-1]:.4f}; held-out {held:.4f}")
    assert hist[-1] < hist[0]
    assert held < 0.9
    # DFGMRES iterations on the Newton system, plain vs corrected, at the continuation's
    # linear tolerance (1e-1) and at a tight one (1e-6)
    its = {}
    for tol in (1e-1, 1e-6):
        sol = DFGMRES(P.dmesh, tol, 200, 1e-3, amg=amg)
        lc.off(amg)
        x0, it_plain = sol.solve(K, s["b"])
        lc.features(K, s["b"])
        lc.correction(amg)
        x1, it_learned = sol.solve(K, s["b"])
        lc.off(amg)
        its[tol] = (it_plain, it_learned)
        r1 = (s["A"] @ x1.cpu().numpy()) - s["b"].cpu().numpy()
        assert np.linalg.norm(r1) <= 1.1 * tol * np.linalg.norm(s["b"].cpu().numpy())
    print(f"DFGMRES iterations (plain, corrected): tol 1e-1 {its[1e-1]}, tol 1e-6 {its[1e-6]}")
    assert its[1e-1][1] <= its[1e-1][0]
    # at tight tolerances the non-symmetric local correction may cost a few iterations
    assert its[1e-6][1] <= its[1e-6][0] + 4


def test_dfgmres_hook_trains_and_solves(system):
    s = system
    P, K = s["P"], s["K"]
    solver = set_linear_solver("DFGMRES_B200", 1e-6, 200, 1e-3, 0, P.dmesh, P.mesh.coord,
                               learned=dict(train_at=0, n_vectors=8, steps=30), cons=P.cons)
    solver.setup_preconditioner(K)
    x, it = solver.solve(K, s["b"])
    lc = solver.learned
    assert lc.trained and lc.info()["adam_steps"] == 30
    g = lc.gate
    print(f"acceptance trial: {g}")
    faster = g["corrected_s"] <= (1.0 - lc.trial_margin) * g["plain_s"]
    assert g["accepted"] == (g["corrected_iterations"] < g["plain_iterations"] and faster)
    assert lc.enabled == g["accepted"] and g["tolerance"] == lc.trial_tolerance
    r = (s["A"] @ x.cpu().numpy()) - s["b"].cpu().numpy()
    assert np.linalg.norm(r) <= 1.1e-6 * np.linalg.norm(s["b"].cpu().numpy())

"""CPU checks of the learned-correction oracle (oracle/learned_ref.py), which the tensor-core
kernels are compared against: BF16 rounding equals torch's round-to-nearest-even
conversion, and the exact (FP64) backward pass and the loss gradient dL/dG agree with
central finite differences."""
import numpy as np
import scipy.sparse as sp
import torch

from oracle import learned_ref as L


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-6, 6, 4000), [0.0, -0.0, 1.0, 1.00390625,
                                                                                    1.005859375, -3.0e38]])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(L.bf16(x), ref)
    bits = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(L.bf16_bits(x), bits)


def test_mlp_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = L.init_params(3, zero_last=False).astype(np.float64)
    n = 40
    X = rng.normal(size=(n, L.NF))
    dG = rng.normal(size=(n, L.NO))

    def f(q):
        Y, _ = L.mlp_forward(q, X, exact=True)
        return float((Y * dG).sum())

    g = L.mlp_backward(p, X, dG, exact=True)
    idx = rng.choice(L.NPARAM, 60, replace=False)
    h = 1e-5
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (f(p + e) - f(p - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_correction_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    n = 30
    B = sp.random(3 * n, 3 * n, density=0.1, random_state=4)
    A = (B @ B.T + sp.eye(3 * n) * 3.0).tocsr()
    Kd = np.stack([A[3 * i:3 * i + 3, 3 * i:3 * i + 3].toarray() for i in range(n)])
    Dinv = L.block_inv(Kd)
    mask = np.ones((n, 3))
    mask[0] = 0.0
    rz = [rng.normal(size=3 * n) for _ in range(3)]
    G = rng.normal(size=(n, L.NO)) * 0.3
    for kind in ("energy", "residual"):
        loss, dG = L.correction_loss(G, Dinv, mask, A, rz, kind)
        h = 1e-6
        for _ in range(40):
            i, k = rng.integers(n), rng.integers(9)
            Gp, Gm = G.copy(), G.copy()
            Gp[i, k] += h
            Gm[i, k] -= h
            fd = (L.correction_loss(Gp, Dinv, mask, A, rz, kind)[0]
                  - L.correction_loss(Gm, Dinv, mask, A, rz, kind)[0]) / (2 * h)
            assert abs(fd - dG[i, k]) <= 1e-6 * max(1.0, abs(fd))
        assert np.all(dG[:, 9:] == 0) and np.all(dG[0] == 0)
    # the energy objective is the exact change of the error's energy norm
    d = np.zeros(3 * n)
    y = np.einsum("nij,nj->ni", Dinv, rz[0].reshape(n, 3))
    d[:] = (np.einsum("nij,nj->ni", G[:, :9].reshape(n, 3, 3), y) * mask).ravel()
    e = np.linalg.solve(A.toarray(), rz[0])
    change = (e - d) @ (A @ (e - d)) - e @ (A @ e)
    assert abs(L.correction_loss(G, Dinv, mask, A, rz[:1], "energy")[0] * float(rz[0] @ y.ravel()) - change) \
        <= 1e-9 * abs(change)


def test_acceptance_trial_rule():
    """The correction is kept only with fewer iterations AND at most (1 - margin) of the plain
    trial time (host logic of LearnedCorrection.decide; no device state involved)."""
    from slope_stability_octave_b200.learned import LearnedCorrection
    lc = LearnedCorrection.__new__(LearnedCorrection)
    lc.trial_margin, lc.trial_tolerance, lc.train_seconds = 0.05, 1e-6, 0.0
    cases = [((30, 25, 1.0, 0.90), True),     # fewer iterations and 10 % faster
             ((30, 25, 1.0, 0.97), False),    # fewer iterations but within the margin
             ((25, 25, 1.0, 0.50), False),    # not fewer iterations
             ((25, 30, 1.0, 0.80), False),
             ((30, 25, None, None), True)]    # untimed trial: iterations alone
    for (ip, ic, tp, tc), want in cases:
        lc.decide(ip, ic, 0.1, t_plain=tp, t_corrected=tc)
        assert lc.gate["accepted"] is want and lc.enabled is want, (ip, ic, tp, tc)
    assert abs(lc.train_seconds - 0.5) < 1e-12

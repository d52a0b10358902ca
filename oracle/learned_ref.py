"""CPU restatement of the learned node-wise V-cycle correction (test infrastructure only).

The correction has no counterpart in the reference (its DFGMRES preconditioner is one
BoomerAMG V-cycle, +LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp:751-796); this module
states the network, its gradient, the node features and the training loss in NumPy so the
tensor-core kernels can be checked against it:

  mlp_forward / mlp_backward   the per-node network 16 -> 64 -> 64 -> 16 (ReLU), with the
                               kernels' BF16 rounding points (features, weights, hidden
                               activations, output gradient and hidden gradients) and
                               FP64 accumulation; ``exact=True`` drops the rounding (for
                               finite-difference checks of the gradient formulas)
  features                     the 16 node features
  correction_loss              the training objective (energy norm of the corrected error, or
                               the residual norm) and dL/dG

Parity is pinned by the finite-difference checks of the FP64 path in the tests (there is no
reference implementation to pin against).
"""
from __future__ import annotations

import numpy as np

NF, NH, NO = 16, 64, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + NF * NH
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH * NO
NPARAM = OFF_B3 + NO


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_bits(x):
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def unpack(p):
    p = np.asarray(p)
    if p.dtype not in (np.float32, np.float64):
        p = p.astype(np.float64)
    W1 = p[OFF_W1:OFF_B1].reshape(NF, NH)
    b1 = p[OFF_B1:OFF_W2]
    W2 = p[OFF_W2:OFF_B2].reshape(NH, NH)
    b2 = p[OFF_B2:OFF_W3]
    W3 = p[OFF_W3:OFF_B3].reshape(NH, NO)
    b3 = p[OFF_B3:NPARAM]
    return W1, b1, W2, b2, W3, b3


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([np.ravel(a) for a in (W1, b1, W2, b2, W3, b3)]).astype(np.float32)


def init_params(seed, zero_last=True):
    """He-uniform first two layers, 0.01 hidden biases, last layer zero (as the library
    initialises, with its own generator: values differ, the distribution is the same)."""
    rng = np.random.default_rng(seed)
    W1 = rng.uniform(-1, 1, (NF, NH)) * np.sqrt(6.0 / NF)
    W2 = rng.uniform(-1, 1, (NH, NH)) * np.sqrt(6.0 / NH)
    W3 = np.zeros((NH, NO)) if zero_last else rng.uniform(-1, 1, (NH, NO)) * np.sqrt(6.0 / NH)
    return pack(W1, np.full(NH, 0.01), W2, np.full(NH, 0.01), W3, np.zeros(NO))


def _r(x, exact):
    return np.asarray(x, np.float64) if exact else bf16(x).astype(np.float64)


def mlp_forward(p, X, exact=False):
    """Network output (n x 16) and the intermediates the backward pass needs."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Xr = _r(X, exact)
    Z1 = Xr @ _r(W1, exact) + b1
    H1 = _r(np.maximum(Z1, 0.0), exact)
    Z2 = H1 @ _r(W2, exact) + b2
    H2 = _r(np.maximum(Z2, 0.0), exact)
    Y = H2 @ _r(W3, exact) + b3
    return Y, dict(X=Xr, Z1=Z1, H1=H1, Z2=Z2, H2=H2)


def mlp_backward(p, X, dG, exact=False):
    """Gradient (NPARAM) of sum_i <dG_i, Y_i> with respect to the parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    _, c = mlp_forward(p, X, exact)
    dY = _r(dG, exact)
    gW3 = c["H2"].T @ dY
    gb3 = dY.sum(0)
    dZ2 = _r((dY @ _r(W3, exact).T) * (c["Z2"] > 0), exact)
    gW2 = c["H1"].T @ dZ2
    gb2 = dZ2.sum(0)
    dZ1 = _r((dZ2 @ _r(W2, exact).T) * (c["Z1"] > 0), exact)
    gW1 = c["X"].T @ dZ1
    gb1 = dZ1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])


def features(Kdiag, mask, coord, res, elem, n_q, branch=None, c_bar=None):
    """Node features (n x 16 float32, before BF16 rounding).

    Kdiag (n x 3 x 3) diagonal blocks; mask (n x 3) 1 free / 0 Dirichlet; coord (3 x n);
    res (n x 3) Newton residual; elem (n_p x n_e) 0-based; branch, c_bar per integration
    point (element-major, n_q per element) or None."""
    n = Kdiag.shape[0]
    n_e = elem.shape[1]
    f = np.zeros((n, NF))
    d = np.abs(np.stack([Kdiag[:, a, a] for a in range(3)], 1))
    dmean = (d * mask).sum() / max(mask.sum(), 1.0)
    rrms = np.sqrt((res ** 2 * mask).sum() / max(mask.sum(), 1.0)) or 1.0
    f[:, 0:3] = np.log10(np.maximum(d, 1e-300) / dmean)
    f[:, 8:11] = np.sign(res / rrms) * np.log1p(np.abs(res / rrms))
    ep = (np.asarray(branch).reshape(n_e, n_q) != 0).mean(1) if branch is not None else np.zeros(n_e)
    ec = np.asarray(c_bar).reshape(n_e, n_q).mean(1) if c_bar is not None else np.zeros(n_e)
    cnt = np.zeros(n)
    ps = np.zeros(n)
    cs = np.zeros(n)
    for k in range(elem.shape[0]):
        np.add.at(cnt, elem[k], 1.0)
        np.add.at(ps, elem[k], ep)
        np.add.at(cs, elem[k], ec)
    has = cnt > 0
    f[has, 3] = ps[has] / cnt[has]
    if c_bar is not None:
        cmean = float(np.mean(c_bar)) or 1.0
        f[has, 11] = np.log(np.maximum(cs[has] / cnt[has], 1e-300) / cmean)
    lo, hi = coord.min(1), coord.max(1)
    span = np.where(hi > lo, hi - lo, 1.0)
    f[:, 4:7] = (2.0 * (coord.T - lo) / span - 1.0)
    mf = mask.sum(1)
    f[:, 7] = (mf == 3).astype(float)
    f[:, 12] = mf / 3.0
    return f.astype(np.float32)


def block_inv(Kdiag):
    out = np.zeros_like(Kdiag)
    det = np.linalg.det(Kdiag)
    ok = np.abs(det) > 0
    out[ok] = np.linalg.inv(Kdiag[ok])
    return out


def correction_loss(G, Dinv, mask, A, rz_list, kind="energy"):
    """L and dL/dG (n x 16, columns 9.. zero) for the correction d = M (G9 Dinv rz).

    kind "residual": L = (1/S) sum |rz - A d|^2 / |rz|^2;
    kind "energy":   L = (1/S) sum (d'A d - 2 d'rz) / (rz' Dinv rz), the change of the
                     error's energy norm |e - d|_A^2 - |e|_A^2 for A e = rz."""
    n = Dinv.shape[0]
    G9 = np.asarray(G, np.float64)[:, :9].reshape(n, 3, 3)
    S = len(rz_list)
    L = 0.0
    dG = np.zeros((n, NO))
    for rz in rz_list:
        rz = np.asarray(rz, np.float64)
        y = np.einsum("nij,nj->ni", Dinv, rz.reshape(n, 3))
        d = (np.einsum("nij,nj->ni", G9, y) * mask).ravel()
        q = A @ d
        e = rz - q
        if kind == "energy":
            w = 1.0 / (S * float(rz @ y.ravel()))
            L += w * float(d @ (q - 2.0 * rz))
            g = e.reshape(n, 3) * mask
        else:
            w = 1.0 / (S * float(rz @ rz))
            L += w * float(e @ e)
            g = (A @ e).reshape(n, 3) * mask
        dG[:, :9] += (-2.0 * w * np.einsum("na,nb->nab", g, y)).reshape(n, 9)
    return L, dG

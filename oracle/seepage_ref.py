"""CPU restatement of the reference's SEEPAGE package and of the 2D P1 -> P2 mesh conversion
(test infrastructure: the GPU path is checked against these functions; nothing in the
product imports them).

  penalty_parameters   +SEEPAGE/penalty_parameters_3D.m:16-47, penalty_parameters_2D.m:16-43
  auxiliary_matrices   +SEEPAGE/auxiliary_matrices_3D.m:52-135, _2D.m (Bw, C, weight as the
                       reference's sparse operators)
  seepage_problem      +SEEPAGE/seepage_problem_3D.m:1-75, seepage_problem_2D.m:1-59
  newton_flow          +SEEPAGE/newton_flow.m:47-186
  midpoints_p2_2d      +MESH/midpoints_P2.m:1-90 (edge midpoints in the reference's numbering,
                       and its boundary list ``surf``, whose every column is [V3; V2; mid]
                       whichever edge the midpoint lies on)
  franz_dam_mesh       +MESH/load_mesh_Franz_dam.m:1-40 on the arrays of meshes/Franz_dam
  franz_dam_seepage_bc slope_stability_2D_Franz_dam_SSR.m:100-128 (Q_w and pw_D)

Linear systems are solved directly (scipy.sparse.linalg.spsolve): the reference's Newton
stops on the relative update 1e-10, so the converged pressure does not depend on the
solver to that level.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

GRHO = 9.81


def penalty_parameters(coord, elem):
    """Per element grho * min edge length / 2; the 3D L34 term adds (z2 - z4)^2, as written in
    penalty_parameters_3D.m:44."""
    coord = np.asarray(coord, np.float64)
    dim = coord.shape[0]
    n_e = elem.shape[1]
    eps = np.zeros(n_e)
    X = [coord[:, elem[i]] for i in range(dim + 1)]
    if dim == 3:
        def L(a, b, zc=None):
            za = X[zc][2] if zc is not None else X[a][2]
            return np.sqrt((X[a][0] - X[b][0]) ** 2 + (X[a][1] - X[b][1]) ** 2 + (za - X[b][2]) ** 2)
        Ls = [L(0, 1), L(0, 2), L(1, 2), L(0, 3), L(1, 3), L(2, 3, zc=1)]
    else:
        def L(a, b):
            return np.sqrt((X[a][0] - X[b][0]) ** 2 + (X[a][1] - X[b][1]) ** 2)
        Ls = [L(0, 1), L(0, 2), L(1, 2)]
    eps[:] = GRHO * np.min(np.vstack(Ls), axis=0) / 2
    return eps


def auxiliary_matrices(elem, dphi, weight, hat):
    """Bw (dim*n_int x n_n; row dim*g + d = d/dx_d at point g) and C (n_int x n_n), as the
    sparse operators of auxiliary_matrices_3D.m:115-133.  dphi: tuple of (n_int, n_p)
    physical gradients; hat: (n_p, n_q) basis values."""
    dim = len(dphi)
    n_p, n_e = elem.shape
    n_q = hat.shape[1]
    n_int = n_e * n_q
    n_n = int(elem.max()) + 1
    cols = np.repeat(elem.T, n_q, axis=0)                       # (n_int, n_p) node of (g, i)
    rows = []
    vals = []
    for d in range(dim):
        rows.append(np.repeat((dim * np.arange(n_int) + d)[:, None], n_p, axis=1))
        vals.append(dphi[d])
    Bw = sp.csr_matrix((np.concatenate([v.ravel() for v in vals]),
                        (np.concatenate([r.ravel() for r in rows]), np.tile(cols.ravel(), dim))),
                       shape=(dim * n_int, n_n))
    vC = np.tile(hat.T, (n_e, 1))                               # (n_int, n_p)
    C = sp.csr_matrix((vC.ravel(), (np.repeat(np.arange(n_int), n_p), cols.ravel())), shape=(n_int, n_n))
    return Bw, C, np.asarray(weight, np.float64)


def _perm(pw_int, eps_int):
    perm = np.ones_like(pw_int)
    der = np.zeros_like(pw_int)
    p1 = (pw_int < eps_int) & (pw_int > 0)
    p2 = pw_int <= 0
    perm[p1] = pw_int[p1] / eps_int[p1]
    perm[p2] = 0
    der[p1] = 1.0 / eps_int[p1]
    return perm, der


def system(pw, Bw, C, K_D, wc, weight, conduct0, q2, eps_int, grho, dim, kappa_mode=2, want_K=True, gq=None):
    """(K, f) of newton_flow.m:88-123 at pw (kappa_mode 0/1: the initial right-hand sides of
    seepage_problem_2D.m / _3D.m with K = K_D).  q2 = Bw y; gq = Bw (grho y) (the E term's
    factor, newton_flow.m:104-105; defaults to grho q2)."""
    n_int = C.shape[0]
    pw_int = C @ pw
    perm, der = _perm(pw_int, eps_int)
    kappa = {0: np.zeros(n_int), 1: np.ones(n_int), 2: perm}[kappa_mode]
    K = None
    if want_K:
        if kappa_mode == 2:
            vE = np.repeat(conduct0 * der * weight, dim) * (grho * q2 if gq is None else gq)
            E = sp.csr_matrix((vE, (np.arange(dim * n_int), np.repeat(np.arange(n_int), dim))),
                              shape=(dim * n_int, n_int))
            K = (K_D + Bw.T @ (E @ C)).tocsr()
        else:
            K = K_D
    q3 = Bw @ pw + grho * np.repeat(kappa, dim) * q2
    f = -(Bw.T @ (np.repeat(wc, dim) * q3))
    return K, f


def seepage_problem(coord, elem, Q_w, pw_D, grho, conduct0, hat, dphi, weight, it_max=50, tol=1e-10):
    """[pw, grad_p, mater_sat, stats] of seepage_problem_3D.m / _2D.m with direct solves."""
    dim = len(dphi)
    n_p, n_e = elem.shape
    n_q = hat.shape[1]
    Q_w = np.asarray(Q_w, bool)
    eps = penalty_parameters(coord, elem)
    eps_int = np.repeat(eps, n_q)
    Bw, C, weight = auxiliary_matrices(elem, dphi, weight, hat)
    wc = weight * conduct0
    Dm = sp.diags(np.repeat(wc, dim))
    K_D = (Bw.T @ Dm @ Bw).tocsr()
    q2 = Bw @ np.asarray(coord[1], np.float64)
    gq = Bw @ (grho * np.asarray(coord[1], np.float64))
    _, f = system(pw_D, Bw, C, K_D, wc, weight, conduct0, q2, eps_int, grho, dim,
                  kappa_mode=1 if dim == 3 else 0, want_K=False)
    pw0 = np.zeros(coord.shape[1])
    pw0[Q_w] = spla.spsolve(K_D[Q_w][:, Q_w].tocsc(), f[Q_w])
    pw_init = pw0 + pw_D
    pw, stats = newton_flow(pw_init, Bw, C, K_D, wc, weight, conduct0, q2, eps_int, grho, dim, Q_w, it_max, tol,
                            gq=gq)
    grad_p = (Bw @ pw).reshape(-1, dim)
    pw_int = C @ pw
    if n_q > 1:
        aver = (pw_int * weight).reshape(n_e, n_q).sum(1) / weight.reshape(n_e, n_q).sum(1)
    else:
        aver = pw_int
    mater_sat = aver >= 0.1 * eps
    return pw, grad_p, mater_sat, dict(stats, eps=eps, aver=aver, pw_init=pw_init)


def newton_flow(pw_init, Bw, C, K_D, wc, weight, conduct0, q2, eps_int, grho, dim, Q_w, it_max=50, tol=1e-10,
                it_damp_max=10, gq=None):
    pw = pw_init.copy()
    it = 0
    norm_ref = max(1.0, np.linalg.norm(pw_init))
    alphas, rel = [], []
    status = "unknown"
    while True:
        it += 1
        K, f = system(pw, Bw, C, K_D, wc, weight, conduct0, q2, eps_int, grho, dim, gq=gq)
        dp = np.zeros_like(pw)
        dp[Q_w] = spla.spsolve(K[Q_w][:, Q_w].tocsc(), f[Q_w])
        criterion = np.linalg.norm(f[Q_w])
        alpha, it_damp = 1.0, 0
        while it_damp < it_damp_max:
            it_damp += 1
            _, fa = system(pw + alpha * dp, Bw, C, K_D, wc, weight, conduct0, q2, eps_int, grho, dim, want_K=False)
            if np.linalg.norm(fa[Q_w]) < criterion:
                break
            alpha /= 2
        if it_damp >= it_damp_max:
            alpha = 0.0
        pw = pw + alpha * dp
        r = np.linalg.norm(dp) / norm_ref
        alphas.append(alpha)
        rel.append(r)
        if r < tol:
            status = "converged"
            break
        if np.isnan(r):
            status = "nan_update"
            break
        if it > it_max:
            status = "max_iterations"
            break
    return pw, dict(iterations=it, alphas=alphas, rel_updates=rel, status=status)


# ------------------------------------------------------------------ 2D P1 -> P2 and the Franz dam


def midpoints_p2_2d(coord, elem):
    """coord_mid (2, n_mid), elem_mid (3, n_e) 0-based node ids, surf (3, n_s) 0-based, in the
    numbering of midpoints_P2.m: element by element, edges V2-V3, V3-V1, V1-V2; a boundary
    edge appends [V3; V2; mid] to surf (for every one of the three edges)."""
    coord = np.asarray(coord, np.float64)
    elem = np.asarray(elem, np.int64)
    n_n = coord.shape[1]
    n_e = elem.shape[1]
    # edge -> elements containing both vertices
    from collections import defaultdict
    owners = defaultdict(list)
    for e in range(n_e):
        v = elem[:, e]
        for a, b in ((1, 2), (2, 0), (0, 1)):
            owners[frozenset((int(v[a]), int(v[b])))].append(e)
    elem_mid = -np.ones((3, n_e), np.int64)
    mids = []
    surf = []
    for i in range(n_e):
        V1, V2, V3 = (int(x) for x in elem[:, i])
        for slot, (P, Qv) in enumerate(((V2, V3), (V3, V1), (V1, V2))):
            if elem_mid[slot, i] >= 0:
                continue
            mids.append((coord[:, P] + coord[:, Qv]) / 2)
            idx = n_n + len(mids) - 1
            elem_mid[slot, i] = idx
            others = [j for j in owners[frozenset((P, Qv))] if j != i]
            if others:
                j = others[0]
                v = elem[:, j]
                if Qv == v[0]:
                    elem_mid[2, j] = idx
                elif Qv == v[1]:
                    elem_mid[0, j] = idx
                else:
                    elem_mid[1, j] = idx
            else:
                surf.append((V3, V2, idx))
    return np.array(mids).T, elem_mid, np.array(surf, np.int64).T


def franz_dam_mesh(coords_p1, elems_p1, materials_1based):
    """load_mesh_Franz_dam.m for elem_type 'P2': 0-based elem (6, n_e), coord (2, n_n),
    Q (2, n_n), mater (0-based), surf (3, n_s)."""
    coord = np.asarray(coords_p1, np.float64).T.copy()
    elem = np.asarray(elems_p1, np.int64).T.copy()
    mater = np.asarray(materials_1based, np.int64).reshape(-1) - 1
    cm, em, surf = midpoints_p2_2d(coord, elem)
    coord = np.hstack([coord, cm])
    elem = np.vstack([elem, em])
    x_max, x_min, y_min = coord[0].max(), coord[0].min(), coord[1].min()
    Q = np.zeros((2, coord.shape[1]), bool)
    Q[0] = (coord[0] > x_min + 0.2) & (coord[1] > y_min + 0.2) & (coord[0] < x_max - 0.2)
    Q[1] = coord[1] > y_min + 0.2
    return coord, elem, Q, mater, surf


def franz_dam_seepage_bc(coord, surf, grho=GRHO):
    """Q_w and pw_D of slope_stability_2D_Franz_dam_SSR.m:100-128."""
    n_n = coord.shape[1]
    Q_D = (coord[1, surf[0]] + coord[1, surf[1]]) / 2 >= -400 + 1e-1
    Q_w = np.ones(n_n, bool)
    Q_w[np.unique(surf[:, Q_D])] = False
    x1, y1 = -82.5, -50.0
    x2, y2 = 172.5, -112.0
    x, y = coord
    pw_D = np.zeros(n_n)
    p1 = (x < x1 + 1e-9) & (y < y1)
    p2 = (x >= x1 + 1e-9) & (x < x2 + 1e-9) & (y < ((y2 - y1) / (x2 - x1)) * (x - x1) + y1)
    p3 = (x >= x2 + 1e-9) & (y < y2)
    pw_D[p1] = grho * (y1 - y[p1])
    pw_D[p2] = grho * (((y2 - y1) / (x2 - x1)) * (x[p2] - x1) + y1 - y[p2])
    pw_D[p3] = grho * (y2 - y[p3])
    return Q_w, pw_D


def homo_slope_seepage_bc(coord, x1=15.0, x2=10.0, x3=15.0, y1=10.0, y2=10.0, y21=2.0, y22=6.0, grho=GRHO):
    """Q_w and pw_D of slope_stability_3D_homo_seepage_SSR.m:108-133 (phreatic line y21 / y22)."""
    x, y = coord[0], coord[1]
    n_n = coord.shape[1]
    Q_w = np.ones(n_n, bool)
    Q_w[x <= 0.001] = False
    Q_w[x >= x1 + x2 + x3 - 0.001] = False
    Q_w[y >= y1 + y2 - 0.001] = False
    Q_w[(y >= y1 - 0.001) & (x >= x1 + x2 - 0.001)] = False
    Q_w[(y >= y1 - 0.001) & (y >= -(y2 / x2) * x + y1 + y2 * (1 + x1 / x2) - 0.001)] = False
    pw_D = np.zeros(n_n)
    x_bar = x1 + (1 - y21 / y2) * x2
    p1 = (x < x_bar) & (y <= -(y22 / x_bar) * x + y1 + y21 + y22)
    p2 = x >= x_bar
    pw_D[p1] = grho * ((y22 / x_bar) * (x_bar - x[p1]) + y1 + y21 - y[p1])
    pw_D[p2] = grho * (y1 + y21 - y[p2])
    return Q_w, pw_D

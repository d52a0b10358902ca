"""ORACLE (test infrastructure): SciPy restatement of the product's AMG preconditioner.

The reference's preconditioner is HYPRE BoomerAMG (+LINEAR_SOLVERS/mex/hypre_boomeramg_mex.cpp),
which is not part of this build (not vendored, cloned from git master at set-up time), so
BoomerAMG parity is unpinned.  The product uses its own smoothed-aggregation AMG; this module
restates that algorithm so its hierarchy and V-cycle can be checked on the CPU:

  aggregate        three-phase aggregation of the block graph (roots with untouched
                   neighbourhoods; leftovers join the most-connected neighbouring aggregate;
                   the rest form their own aggregates); optional strength filter
  tentative        per-aggregate thin QR of the near-null space (two-pass Gram-Schmidt)
  Hierarchy        P = T - omega D^-1 A T (omega = 4/3 / lambda_max(D^-1 A), power iteration
                   from the same deterministic start vector), A_c = P' A P, dense inverse on the
                   coarsest level, Chebyshev(degree) smoothing on D^-1 A over
                   [lambda_max/ratio, 1.1 lambda_max], V(1,1) cycle
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def block_graph(A, b):
    """Block pattern (rp, col) of a scipy matrix with b x b blocks."""
    Ab = sp.bsr_matrix(A, blocksize=(b, b))
    Ab.sort_indices()
    return Ab.indptr.astype(np.int64), Ab.indices.astype(np.int64)


def strength_graph(A, b, theta):
    """Block rows keep (i, j) when ||A_ij||_F >= theta * sqrt(||A_ii||_F ||A_jj||_F) (and i == j)."""
    Ab = sp.bsr_matrix(A, blocksize=(b, b))
    Ab.sort_indices()
    n = Ab.shape[0] // b
    nrm = np.sqrt((Ab.data ** 2).sum(axis=(1, 2)))
    rows = np.repeat(np.arange(n), np.diff(Ab.indptr))
    diag = np.zeros(n)
    dm = rows == Ab.indices
    diag[rows[dm]] = nrm[dm]
    keep = (nrm >= theta * np.sqrt(diag[rows] * diag[Ab.indices])) | dm
    G = sp.csr_matrix((np.ones(keep.sum()), (rows[keep], Ab.indices[keep])), shape=(n, n))
    G.sort_indices()
    return G.indptr.astype(np.int64), G.indices.astype(np.int64)


def aggregate(rp, col, active):
    n = rp.size - 1
    agg = -np.ones(n, np.int64)
    na = 0
    for i in range(n):
        if not active[i] or agg[i] >= 0:
            continue
        nb = col[rp[i]:rp[i + 1]]
        nb = nb[active[nb]]
        if np.any(agg[nb] >= 0):
            continue
        agg[nb] = na
        agg[i] = na
        na += 1
    add = -np.ones(n, np.int64)
    for i in range(n):
        if not active[i] or agg[i] >= 0:
            continue
        a = agg[col[rp[i]:rp[i + 1]]]
        a = a[a >= 0]
        if a.size:
            vals, cnt = np.unique(a, return_counts=True)
            # most connections; ties -> first seen in row order
            best = -1
            bestc = 0
            for x in col[rp[i]:rp[i + 1]]:
                ax = agg[x]
                if ax < 0:
                    continue
                c = cnt[np.searchsorted(vals, ax)]
                if c > bestc:
                    bestc, best = c, ax
            add[i] = best
    agg[add >= 0] = add[add >= 0]
    for i in range(n):
        if not active[i] or agg[i] >= 0:
            continue
        nb = col[rp[i]:rp[i + 1]]
        nb = nb[active[nb] & (agg[nb] < 0)]
        agg[nb] = na
        agg[i] = na
        na += 1
    return agg, na


def tentative(agg, na, B, b, k):
    """Returns T (n*b x na*k, sparse: node rows hold a b x k block in their aggregate's
    column block), the coarse near-null space Bc (na*k x k) and dead coarse DOFs."""
    n = agg.size
    Tn = np.zeros((n * b, k))
    Bc = np.zeros((na * k, k))
    dead = np.zeros(na * k, bool)
    for a in range(na):
        mem = np.nonzero(agg == a)[0]
        rows = (mem[:, None] * b + np.arange(b)[None, :]).ravel()
        Qm = B[rows].copy()
        R = np.zeros((k, k))
        scale = np.abs(Qm).max() if Qm.size else 0.0
        for c in range(k):
            n0 = np.linalg.norm(Qm[:, c])
            for _ in range(2):
                for c2 in range(c):
                    h = Qm[:, c2] @ Qm[:, c]
                    Qm[:, c] -= h * Qm[:, c2]
                    R[c2, c] += h
            nr = np.linalg.norm(Qm[:, c])
            if nr <= 1e-10 * max(n0, scale * 1e-3) or nr == 0.0:
                Qm[:, c] = 0.0
                R[c, :] = 0.0
                dead[a * k + c] = True
                continue
            R[c, c] = nr
            Qm[:, c] /= nr
        Tn[rows] = Qm
        Bc[a * k:(a + 1) * k] = R
    node = np.repeat(np.arange(n), b)
    ok = agg[node] >= 0
    rr = np.repeat(np.nonzero(ok)[0], k)
    cc = (agg[node[ok]][:, None] * k + np.arange(k)[None, :]).ravel()
    T = sp.csr_matrix((Tn[ok].ravel(), (rr, cc)), shape=(n * b, na * k))
    return T, Bc, dead


def _filtered(A, b, rp, col):
    """A with the blocks outside the strength graph (rp, col) removed and their row sums
    added to the diagonal block's diagonal (so A_F keeps A's action on constants)."""
    Ab = sp.bsr_matrix(A, blocksize=(b, b))
    Ab.sort_indices()
    n = Ab.shape[0] // b
    data = Ab.data.copy()
    for i in range(n):
        keep = set(col[rp[i]:rp[i + 1]].tolist())
        dpos = None
        lump = np.zeros(b)
        for p in range(Ab.indptr[i], Ab.indptr[i + 1]):
            j = Ab.indices[p]
            if j == i:
                dpos = p
            elif j not in keep:
                lump += data[p].sum(axis=1)
                data[p] = 0.0
        if dpos is not None:
            data[dpos] += np.diag(lump)
    F = sp.bsr_matrix((data, Ab.indices, Ab.indptr), shape=Ab.shape).tocsr()
    F.eliminate_zeros()
    return F


def _block_dinv(A, b):
    n = A.shape[0] // b
    D = np.zeros((n, b, b))
    Ab = sp.bsr_matrix(A, blocksize=(b, b))
    Ab.sort_indices()
    for i in range(n):
        for p in range(Ab.indptr[i], Ab.indptr[i + 1]):
            if Ab.indices[p] == i:
                D[i] = Ab.data[p]
    return np.linalg.inv(D)


def _init_vec(n):
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        h = i * np.uint64(0x9E3779B97F4A7C15) + np.uint64(0x632BE59BD9B4E019)
        h ^= h >> np.uint64(31)
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(29)
    return 0.5 + (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class Hierarchy:
    def __init__(self, A, B, b, fixed=None, coarse_size=1200, max_levels=10, cheb_degree=3, cheb_ratio=10.0,
                 power_its=10, omega_scale=4.0 / 3.0, theta=0.0, theta_coarse=None, filtered_smoothing=False):
        self.deg, self.ratio = cheb_degree, cheb_ratio
        A = sp.csr_matrix(A)
        n = A.shape[0] // b
        nns = B.shape[1]
        B = B.copy()
        active = np.ones(n, bool)
        if fixed is not None:
            B[fixed] = 0.0
            active = ~fixed.reshape(n, b).all(axis=1)
        self.levels = []
        dead = None
        while True:
            lev = dict(A=A, b=b)
            if dead is not None:
                lev["dead"] = dead
            lev["Dinv"] = _block_dinv(A, b)
            self.levels.append(lev)
            ndof = A.shape[0]
            last = ndof <= coarse_size or len(self.levels) >= max_levels
            na = 0
            if not last:
                th = theta if (len(self.levels) == 1 or theta_coarse is None) else theta_coarse
                rp, col = strength_graph(A, b, th) if th > 0 else block_graph(A, b)
                agg, na = aggregate(rp, col, active)
            if last or na == 0 or na * nns >= ndof * 3 // 4:
                lev["Ainv"] = np.linalg.inv(A.toarray())
                break
            T, Bc, dead = tentative(agg, na, B, b, nns)
            lev["agg"] = agg
            lev["T"] = T
            lev["dead_next"] = dead
            # lambda_max(D^-1 A) by power iteration
            v = _init_vec(ndof)
            lmax = 1.0
            for _ in range(power_its):
                w = self.dinv(lev, A @ v)
                lmax = np.linalg.norm(w) or 1.0
                v = w / lmax
            lev["lmax"] = lmax
            Ts = T
            As = A
            if filtered_smoothing and th > 0:
                As = _filtered(A, b, rp, col)
            AT = As @ Ts
            P = Ts - (oscale := omega_scale / lmax) * self._dinv_mat(lev, AT)
            lev["P"] = sp.csr_matrix(P)
            Ac = (P.T @ A @ P).tocsr()
            Ac = Ac.tolil()
            for d in np.nonzero(dead)[0]:
                Ac[d, :] = 0
                Ac[:, d] = 0
                Ac[d, d] = 1.0
            A = Ac.tocsr()
            b = nns
            B = Bc
            active = ~dead.reshape(na, nns).all(axis=1)

    def update(self, A, power_its=10, omega_scale=4.0 / 3.0):
        """Numeric set-up for new values of the level-0 matrix on the kept aggregates and
        tentative prolongators (what the device's sg_amg_update redoes per value update):
        block inverses, lambda_max, P = T - omega D^-1 A T, A_c = P' A P with identity on dead
        coarse DOFs, the coarsest inverse."""
        A = sp.csr_matrix(A)
        for l, lev in enumerate(self.levels):
            lev["A"] = A
            lev["Dinv"] = _block_dinv(A, lev["b"])
            if "T" not in lev:
                lev["Ainv"] = np.linalg.inv(A.toarray())
                break
            v = _init_vec(A.shape[0])
            lmax = 1.0
            for _ in range(power_its):
                w = self.dinv(lev, A @ v)
                lmax = np.linalg.norm(w) or 1.0
                v = w / lmax
            lev["lmax"] = lmax
            P = (lev["T"] - (omega_scale / lmax) * self._dinv_mat(lev, A @ lev["T"])).tocsr()
            lev["P"] = P
            dead = lev["dead_next"]
            keep = sp.diags((~dead).astype(float))
            A = (keep @ (P.T @ A @ P) @ keep + sp.diags(dead.astype(float))).tocsr()
        return self

    @classmethod
    def from_levels(cls, mats, prolongators, blocks, cheb_degree=3, cheb_ratio=10.0, power_its=10):
        """V-cycle on a given hierarchy: mats[l] (level matrices), prolongators[l] (l < L-1);
        smoother data (block inverse, lambda_max) recomputed the same way as the device."""
        self = cls.__new__(cls)
        self.deg, self.ratio = cheb_degree, cheb_ratio
        self.levels = []
        for l, A in enumerate(mats):
            lev = dict(A=sp.csr_matrix(A), b=blocks[l])
            lev["Dinv"] = _block_dinv(lev["A"], blocks[l])
            if l == len(mats) - 1:
                lev["Ainv"] = np.linalg.inv(lev["A"].toarray())
            else:
                v = _init_vec(A.shape[0])
                lmax = 1.0
                for _ in range(power_its):
                    w = self.dinv(lev, lev["A"] @ v)
                    lmax = np.linalg.norm(w) or 1.0
                    v = w / lmax
                lev["lmax"] = lmax
                lev["P"] = sp.csr_matrix(prolongators[l])
            self.levels.append(lev)
        return self

    def dinv(self, lev, x):
        b = lev["b"]
        return np.einsum("nab,nb->na", lev["Dinv"], x.reshape(-1, b)).ravel()

    def _dinv_mat(self, lev, M):
        b = lev["b"]
        n = lev["A"].shape[0] // b
        D = sp.bsr_matrix((lev["Dinv"], np.arange(n), np.arange(n + 1)), shape=(n * b, n * b)).tocsr()
        return D @ M

    def smooth(self, lev, x, rhs, x_zero):
        lmax = lev["lmax"]
        hi, lo = 1.1 * lmax, lmax / self.ratio
        theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
        sigma = theta / delta
        rho = 1.0 / sigma
        d = None
        for k in range(self.deg):
            r = rhs if (x_zero and k == 0) else rhs - lev["A"] @ x
            s = self.dinv(lev, r)
            if k == 0:
                d = s / theta
            else:
                rn = 1.0 / (2 * sigma - rho)
                d = rn * rho * d + 2 * rn / delta * s
                rho = rn
            x = d.copy() if (x_zero and k == 0) else x + d
        return x

    def vcycle(self, r, l=0):
        lev = self.levels[l]
        if "Ainv" in lev:
            return lev["Ainv"] @ r
        x = self.smooth(lev, None, r, True)
        res = r - lev["A"] @ x
        xc = self.vcycle(lev["P"].T @ res, l + 1)
        x = x + lev["P"] @ xc
        return self.smooth(lev, x, r, False)

"""ORACLE (test infrastructure): SciPy restatement of the Octave layer of CONSTITUTIVE.m.

Follows Beremi/slope_stability_octave, slope_stability/:
  build_B              +ASSEMBLY/elastic_stiffness_matrix_3D.m:103-132 / _2D.m (sparse B;
                       like Octave's sparse(), exact zeros are not stored)
  init_K_r_pattern     +CONSTITUTIVE_PROBLEM/CONSTITUTIVE.m:393-464 (maximal symbolic pattern
                       of spones(B_Q)' spones(D) spones(B_Q), symmetrised; entries in the
                       column-major order of Octave's find; elastic values; transpose_perm)
  build_scatter_map    CONSTITUTIVE.m:582-635 (1-based int64, 0 = Dirichlet)
  build_K_r_QQ_vals    CONSTITUTIVE.m:515-532 (r-blend and symmetrisation)
  build_F              CONSTITUTIVE.m:268-285 (F = B' (w .* S))
  strain               CONSTITUTIVE.m:218 (E = B U)

Replicated quirk: for n_strain == 3 (2D) the reference builds IOTA = [1;1;1], so VOL is the
all-ones 3x3 matrix and DS_elast couples the shear entry (CONSTITUTIVE.m:413-422).  The
elastic values V_elast_QQ here follow that arithmetic exactly.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import native


def build_B(dim, elem, n_n, dphi):
    """Sparse strain-displacement matrix (n_strain*n_int, dim*n_n), CSR.
    dphi: tuple of (n_int, n_p) arrays; elem (n_p, n_e) 0-based."""
    n_p, n_e = elem.shape
    n_int = dphi[0].shape[0]
    n_q = n_int // n_e
    ns = 6 if dim == 3 else 3
    rows, cols, vals = [], [], []
    node = np.repeat(elem.T, n_q, axis=0)              # (n_int, n_p) node of local i at point g
    g = np.arange(n_int)[:, None]
    if dim == 3:
        d1, d2, d3 = dphi
        table = [(0, 0, d1), (3, 0, d2), (5, 0, d3),
                 (1, 1, d2), (3, 1, d1), (4, 1, d3),
                 (2, 2, d3), (4, 2, d2), (5, 2, d1)]
    else:
        d1, d2 = dphi
        table = [(0, 0, d1), (2, 0, d2), (1, 1, d2), (2, 1, d1)]
    for a, comp, d in table:
        rows.append((ns * g + a) * np.ones_like(node))
        cols.append(dim * node + comp)
        vals.append(d)
    r = np.concatenate([x.ravel() for x in rows])
    c = np.concatenate([x.ravel() for x in cols])
    v = np.concatenate([x.ravel() for x in vals])
    B = sp.coo_matrix((v, (r, c)), shape=(ns * n_int, dim * n_n)).tocsr()
    B.sum_duplicates()
    B.eliminate_zeros()
    return B


def _block_diag_D(ns, n_int, vals):
    """Sparse block-diagonal D with (ns x ns) column-major blocks vals (n_int, ns*ns)."""
    g = np.arange(n_int)
    a = np.tile(np.arange(ns), ns)           # row within block for k = a + ns*b
    b = np.repeat(np.arange(ns), ns)
    rows = (ns * g[:, None] + a[None, :]).ravel()
    cols = (ns * g[:, None] + b[None, :]).ravel()
    return sp.csr_matrix((np.asarray(vals).ravel(), (rows, cols)), shape=(ns * n_int, ns * n_int))


def elastic_DS(dim, shear, bulk):
    """DS_elast of CONSTITUTIVE.m:413-422 (including the 2D IOTA quirk)."""
    ns = 6 if dim == 3 else 3
    iota = np.zeros(ns)
    iota[:3] = 1.0  # [1;1;1; zeros(ns-3,1)] -> all ones when ns == 3
    VOL = np.outer(iota, iota)
    if ns == 6:
        DEV = np.diag([1, 1, 1, 0.5, 0.5, 0.5]) - VOL / 3
    else:
        DEV = np.diag([1, 1, 0.5]) - VOL / 3
    return 2 * DEV.ravel(order="F")[None, :] * shear[:, None] + VOL.ravel(order="F")[None, :] * bulk[:, None]


class OctavePattern:
    """Literal restatement of init_K_r_pattern + build_scatter_map for one mesh."""

    def __init__(self, dim, elem, n_n, dphi, weight, Q, shear, bulk):
        self.dim = dim
        self.ns = 6 if dim == 3 else 3
        self.elem = elem
        self.n_n = n_n
        self.weight = weight
        self.n_int = weight.size
        self.B = build_B(dim, elem, n_n, dphi)
        self.Q_flat = np.nonzero(Q.T.ravel())[0]            # Octave Q(:) is column-major of (dim, n_n)
        self.n_Q = self.Q_flat.size
        B_Q = self.B[:, self.Q_flat].tocsc()
        self.B_Q = B_Q
        DS_el = elastic_DS(dim, shear, bulk)
        self.DS_elast = DS_el
        D_e = _block_diag_D(self.ns, self.n_int, weight[:, None] * DS_el)
        K_el = (B_Q.T @ D_e @ B_Q).tocsc()
        K_el = ((K_el + K_el.T) / 2).tocsc()
        Bp = B_Q.copy()
        Bp.data[:] = 1.0
        Dp = _block_diag_D(self.ns, self.n_int, np.ones((self.n_int, self.ns * self.ns)))
        Ks = (Bp.T @ Dp @ Bp).tocsc()
        Ks = (Ks + Ks.T).tocsc()
        Ks.sort_indices()
        # find(): column-major order -> iterate CSC columns
        J = np.repeat(np.arange(self.n_Q), np.diff(Ks.indptr))
        I = Ks.indices.copy()
        self.ref_I = I.astype(np.int64) + 1
        self.ref_J = J.astype(np.int64) + 1
        self.nnz = I.size
        K_el.sort_indices()
        self.V_elast = np.asarray(K_el[I, J]).ravel()
        # transpose_perm: position of (J, I) in the list
        key = I.astype(np.int64) * self.n_Q + J
        tkey = J.astype(np.int64) * self.n_Q + I
        order = np.argsort(key)
        pos = np.searchsorted(key[order], tkey)
        self.transpose_perm = order[pos] + 1                   # 1-based like Octave
        self._key_sorted = key[order]
        self._order = order

    def lookup(self, rows, cols):
        """1-based pattern index of (rows, cols) (0-based free-DOF indices), 0 if absent."""
        k = rows.astype(np.int64) * self.n_Q + cols
        pos = np.searchsorted(self._key_sorted, k)
        pos = np.minimum(pos, self._key_sorted.size - 1)
        hit = self._key_sorted[pos] == k
        return np.where(hit, self._order[pos] + 1, 0)

    def scatter_map(self):
        """build_scatter_map: (n_e, n_ld^2) int64; column-major local (ii + n_ld*jj) ->
        1-based index k with ref_I[k] = dof(ii), ref_J[k] = dof(jj); 0 if Dirichlet."""
        dim, elem = self.dim, self.elem
        n_p, n_e = elem.shape
        nl = dim * n_p
        free_idx = -np.ones(dim * self.n_n, np.int64)
        free_idx[self.Q_flat] = np.arange(self.n_Q)
        ldof = (dim * elem.T[:, :, None] + np.arange(dim)[None, None, :]).reshape(n_e, nl)
        f = free_idx[ldof]                                    # (n_e, nl)
        rows = np.repeat(f[:, :, None], nl, axis=2)            # ii
        cols = np.repeat(f[:, None, :], nl, axis=1)            # jj
        ok = (rows >= 0) & (cols >= 0)
        m = np.zeros((n_e, nl, nl), np.int64)
        m[ok] = self.lookup(rows[ok], cols[ok])
        # column-major flatten of (ii, jj): index ii + nl*jj
        return np.ascontiguousarray(m.transpose(0, 2, 1).reshape(n_e, nl * nl))

    def K_r_values(self, V_tang, r):
        V = r * self.V_elast + (1 - r) * V_tang
        return (V + V[self.transpose_perm - 1]) / 2

    def assemble_tangent_global(self, DS):
        """build_K_tangent_QQ_vals_global: B_Q' D_t B_Q at the pattern (CONSTITUTIVE.m:503-513)."""
        D_t = _block_diag_D(self.ns, self.n_int, self.weight[:, None] * DS)
        K = (self.B_Q.T @ D_t @ self.B_Q).tocsr()
        return np.asarray(K[self.ref_I - 1, self.ref_J - 1]).ravel()

    def strain(self, U):
        """E = B U; U (dim, n_n) -> (n_int, ns)."""
        return (self.B @ U.T.ravel()).reshape(self.n_int, self.ns)

    def force(self, S):
        """F = B' (w .* S(1:ns,:)) -> (dim, n_n)."""
        ws = (self.weight[:, None] * S[:, : self.ns]).ravel()
        return (self.B.T @ ws).reshape(self.n_n, self.dim).T


def assemble_via_oracle(pat: OctavePattern, dphi, DS, n_q):
    smap = pat.scatter_map()
    d3 = dphi[2] if pat.dim == 3 else None
    return native.assemble(pat.dim, dphi[0], dphi[1], d3, DS, pat.weight, smap, n_q, pat.nnz), smap

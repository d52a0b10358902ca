"""Host-side discretisation set-up (inputs of the Newton-step hot path).

These routines run once per mesh on the host, in NumPy, and produce the arrays the
device path consumes: P2 meshes, quadrature, reference-element gradients, physical
gradients ``DPhi`` and weights ``WEIGHT``, per-point material fields and the gravity
load vector.  They restate the reference's set-up layer:

=====================  ====================================================================
function               reference (Beremi/slope_stability_octave, slope_stability/...)
=====================  ====================================================================
mesh_p2_2d             +MESH/mesh_P2_2D.m:1-263 (trapezoidal slope, P2 triangles)
mesh_p2_3d             +MESH/mesh_P2_3D.m:1-420 (extruded slope, 6 P2 tets per cell)
mesh_p2_box            the same cell split on a plain box (no slope transform)
quadrature_*           +ASSEMBLY/quadrature_volume_{2,3}D.m (P2 rules, constants verbatim)
local_basis_*          +ASSEMBLY/local_basis_volume_{2,3}D.m (P2 bases and gradients)
geometry_3d / _2d      +ASSEMBLY/elastic_stiffness_matrix_{3,2}D.m:49-96 (DPhi, WEIGHT)
materials              +ASSEMBLY/heterogenous_materials.m:51-86
gravity_load           +ASSEMBLY/vector_volume_{3,2}D.m:39-62
=====================  ====================================================================

Layouts: ``coord`` (dim, n_n); ``elem`` (n_p, n_e) 0-based int32; ``Q`` (dim, n_n) bool
free-DOF mask; per-point arrays are flat (n_int,) with point ``g = e*n_q + q``;
``DPhi`` arrays are (n_int, n_p), i.e. the reference's n_p x n_int column-major memory.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# ----------------------------------------------------------------- quadrature


def quadrature_p2_tet():
    """11-point rule of +ASSEMBLY/quadrature_volume_3D.m:39-42 (negative centroid weight).
    The decimal constants are the reference's, kept verbatim so weights match exactly."""
    a, b = 0.0714285714285714, 0.785714285714286
    c, d = 0.399403576166799, 0.100596423833201
    xi = np.array([
        [0.25, a, b, a, a, c, d, d, c, c, d],
        [0.25, a, a, b, a, d, c, d, c, d, c],
        [0.25, a, a, a, b, d, d, c, d, c, c],
    ])
    wf = np.array([-0.013155555555555] + [0.007622222222222] * 4 + [0.024888888888888] * 6)
    return xi, wf


def quadrature_p2_tri():
    """7-point rule of +ASSEMBLY/quadrature_volume_2D.m:24-33 (constants verbatim)."""
    xi = np.array([
        [0.1012865073235, 0.7974269853531, 0.1012865073235, 0.4701420641051, 0.4701420641051,
         0.0597158717898, 1.0 / 3.0],
        [0.1012865073235, 0.1012865073235, 0.7974269853531, 0.0597158717898, 0.4701420641051,
         0.4701420641051, 1.0 / 3.0],
    ])
    wf = np.array([0.1259391805448, 0.1259391805448, 0.1259391805448, 0.1323941527885,
                   0.1323941527885, 0.1323941527885, 0.225]) / 2
    return xi, wf


def local_basis_p2_tet(xi):
    """P2 tet basis (vertices, then edges 01,12,02,13,23,03); local_basis_volume_3D.m:51-104."""
    x1, x2, x3 = xi
    x0 = 1.0 - x1 - x2 - x3
    z = np.zeros_like(x1)
    hat = np.array([x0 * (2 * x0 - 1), x1 * (2 * x1 - 1), x2 * (2 * x2 - 1), x3 * (2 * x3 - 1),
                    4 * x0 * x1, 4 * x1 * x2, 4 * x0 * x2, 4 * x1 * x3, 4 * x2 * x3, 4 * x0 * x3])
    d1 = np.array([-4 * x0 + 1, 4 * x1 - 1, z, z, 4 * (x0 - x1), 4 * x2, -4 * x2, 4 * x3, z, -4 * x3])
    d2 = np.array([-4 * x0 + 1, z, 4 * x2 - 1, z, -4 * x1, 4 * x1, 4 * (x0 - x2), z, 4 * x3, -4 * x3])
    d3 = np.array([-4 * x0 + 1, z, z, 4 * x3 - 1, -4 * x1, z, -4 * x2, 4 * x1, 4 * x2, 4 * (x0 - x3)])
    return hat, d1, d2, d3


def local_basis_p2_tri(xi):
    """P2 triangle basis (vertices, then edges 12, 02, 01); local_basis_volume_2D.m."""
    x1, x2 = xi
    x0 = 1.0 - x1 - x2
    z = np.zeros_like(x1)
    hat = np.array([x0 * (2 * x0 - 1), x1 * (2 * x1 - 1), x2 * (2 * x2 - 1), 4 * x1 * x2, 4 * x0 * x2, 4 * x0 * x1])
    d1 = np.array([-4 * x0 + 1, 4 * x1 - 1, z, 4 * x2, -4 * x2, 4 * (x0 - x1)])
    d2 = np.array([-4 * x0 + 1, z, 4 * x2 - 1, 4 * x1, 4 * (x0 - x2), -4 * x1])
    return hat, d1, d2


# ----------------------------------------------------------------- meshes

# Six P2 tets per hexahedral cell: corner labels 1..8 and edge midpoints "ab".
# Local order per tet: 4 vertices, then edges 01, 12, 02, 13, 23, 03
# (+MESH/mesh_P2_3D.m:210-219).
_CORNER = {1: (0, 0, 0), 2: (2, 0, 0), 3: (2, 2, 0), 4: (0, 2, 0),
           5: (0, 0, 2), 6: (2, 0, 2), 7: (2, 2, 2), 8: (0, 2, 2)}
_TETS = [(1, 2, 4, 6), (1, 4, 5, 6), (4, 5, 6, 8), (2, 3, 4, 6), (3, 6, 7, 4), (4, 6, 7, 8)]
_EDGES = [(0, 1), (1, 2), (0, 2), (1, 3), (2, 3), (0, 3)]


def _tet_offsets():
    """(6, 10, 3) doubled-grid offsets of the 10 nodes of each of the 6 tets of a cell."""
    off = np.zeros((6, 10, 3), np.int64)
    for t, verts in enumerate(_TETS):
        pts = [np.array(_CORNER[v]) for v in verts]
        for a in range(4):
            off[t, a] = pts[a]
        for m, (a, b) in enumerate(_EDGES):
            off[t, 4 + m] = (pts[a] + pts[b]) // 2
    return off


@dataclass
class Mesh:
    """A P2 mesh with its Dirichlet mask.  ``coord`` (dim, n_n), ``elem`` (n_p, n_e) 0-based."""
    coord: np.ndarray
    elem: np.ndarray
    Q: np.ndarray
    info: dict = field(default_factory=dict)

    @property
    def dim(self):
        return self.coord.shape[0]

    @property
    def n_n(self):
        return self.coord.shape[1]

    @property
    def n_e(self):
        return self.elem.shape[1]


def _cells_to_elems(cells, node_id):
    """cells: (n_cell, 3) doubled-grid corner (i0, j0, k0) in enumeration order.
    node_id(i, j, k) -> node number.  Returns elem (10, 6*n_cell)."""
    off = _tet_offsets()
    ijk = cells[:, None, None, :] + off[None, :, :, :]          # (n_cell, 6, 10, 3)
    ids = node_id(ijk[..., 0], ijk[..., 1], ijk[..., 2])       # (n_cell, 6, 10)
    return ids.reshape(-1, 10).T.astype(np.int32).copy()


def mesh_p2_3d(N_h, x1, x2, x3, y1, y2, z):
    """Extruded 3D slope, +MESH/mesh_P2_3D.m:1-420 (coordinates :64-82, split :210-219,
    Dirichlet mask :415-418).  Lengths in m; N_h = cells per metre (integer)."""
    N_x = int(round((x1 + x2 + x3) * N_h))
    N_y = int(round((y1 + y2) * N_h))
    N_z = int(round(z * N_h))
    N1_x = int(round(x1 * N_h))
    N2_x = N_x - N1_x
    N1_y = int(round(y1 * N_h))
    N2_y = N_y - N1_y
    Lx = x1 + x2 + x3
    nx_l, ny_l, nz = 2 * N_x + 1, 2 * N1_y + 1, 2 * N_z + 1
    nx_u, ny_u = 2 * N2_x + 1, 2 * N2_y
    n_low = nx_l * ny_l * nz
    n_n = n_low + nx_u * ny_u * nz

    cx = np.linspace(0.0, Lx, 2 * N_x + 1)
    cy = np.linspace(0.0, y1 + y2, 2 * N_y + 1)
    cz = np.linspace(0.0, z, 2 * N_z + 1)
    # lower box, x mirrored: x = Lx - cx
    K, J, I = np.meshgrid(np.arange(nz), np.arange(ny_l), np.arange(nx_l), indexing="ij")
    xl = Lx - cx[I.ravel()]
    yl = cy[J.ravel()]
    zl = cz[K.ravel()]
    # upper part: width shrinks linearly with the height above the base layer
    K, J, I = np.meshgrid(np.arange(nz), np.arange(ny_u), np.arange(nx_u), indexing="ij")
    s = np.linspace(-x2 - x3, 0.0, nx_u)[I.ravel()]
    eta = cy[1 + J.ravel()]
    cyx = Lx + s * (1.0 - x2 / ((x2 + x3) * y2) * eta)
    xu = Lx - cyx
    yu = cy[2 * N1_y + 1 + J.ravel()]
    zu = cz[K.ravel()]
    coord = np.vstack([np.concatenate([xl, xu]), np.concatenate([yl, yu]), np.concatenate([zl, zu])])

    def node_id(i, j, k):
        low = j <= 2 * N1_y
        idl = i + nx_l * (j + ny_l * k)
        idu = n_low + (i - 2 * N1_x) + nx_u * ((j - 2 * N1_y - 1) + ny_u * k)
        return np.where(low, idl, idu)

    cells = []
    for k0 in range(0, 2 * N_z, 2):
        for j0 in range(0, 2 * N_y, 2):
            i_lo = 0 if j0 < 2 * N1_y else 2 * N1_x
            i0 = np.arange(i_lo, 2 * N_x, 2)
            cells.append(np.stack([i0, np.full_like(i0, j0), np.full_like(i0, k0)], 1))
    cells = np.concatenate(cells)
    elem = _cells_to_elems(cells, node_id)

    x, y, zz = coord
    Q = np.zeros((3, n_n), bool)
    Q[0] = (x > 0) & (y > 0) & (x < Lx)
    Q[1] = y > 0
    Q[2] = (zz > 0) & (y > 0) & (zz < z)
    return Mesh(coord, elem, Q, dict(kind="slope3d", N_h=N_h, dims=(x1, x2, x3, y1, y2, z)))


def mesh_p2_box(nx, ny, nz, h=1.0):
    """Structured box of nx*ny*nz cells of size h, each split into 6 P2 tets exactly as in
    mesh_P2_3D.m (no slope transform).  Bottom (y=0) fixed, lateral faces on rollers."""
    gx, gy, gz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    K, J, I = np.meshgrid(np.arange(gz), np.arange(gy), np.arange(gx), indexing="ij")
    coord = np.vstack([I.ravel() * (h / 2), J.ravel() * (h / 2), K.ravel() * (h / 2)])

    def node_id(i, j, k):
        return i + gx * (j + gy * k)

    K, J, I = np.meshgrid(np.arange(0, 2 * nz, 2), np.arange(0, 2 * ny, 2), np.arange(0, 2 * nx, 2), indexing="ij")
    cells = np.stack([I.ravel(), J.ravel(), K.ravel()], 1)
    elem = _cells_to_elems(cells, node_id)
    x, y, z = coord
    Lx, Lz = nx * h, nz * h
    Q = np.zeros((3, coord.shape[1]), bool)
    Q[0] = (x > 0) & (y > 0) & (x < Lx)
    Q[1] = y > 0
    Q[2] = (z > 0) & (y > 0) & (z < Lz)
    return Mesh(coord, elem, Q, dict(kind="box", cells=(nx, ny, nz), h=h))


def mesh_p2_2d(h, x1, x2, x3, y1, y2):
    """2D trapezoidal slope with P2 triangles, +MESH/mesh_P2_2D.m:1-263 (BC :259-261)."""
    Nx12 = int(round((x1 + x2) / h))
    Nx3 = int(round(x3 / h))
    Nx = Nx12 + Nx3
    Ny1 = int(round(y1 / h))
    Ny2 = int(round(y2 / h))
    Ny = Ny1 + Ny2
    cx = np.concatenate([np.linspace(0, x1 + x2, 2 * Nx12 + 1), np.linspace(x1 + x2, x1 + x2 + x3, 2 * Nx3 + 1)[1:]])
    cy = np.concatenate([np.linspace(0, y1, 2 * Ny1 + 1), np.linspace(y1, y1 + y2, 2 * Ny2 + 1)[1:]])
    C = -np.ones((2 * Nx + 1, 2 * Ny + 1), np.int64)
    xs, ys = [], []
    n = 0
    for j in range(2 * Ny1 + 1):
        C[:, j] = np.arange(n, n + 2 * Nx + 1)
        xs.append(cx)
        ys.append(np.full(2 * Nx + 1, cy[j]))
        n += 2 * Nx + 1
    for j in range(2 * Ny1 + 1, 2 * Ny + 1):
        x_max = x1 + x2 * (y1 + y2 - cy[j]) / y2
        C[: 2 * Nx12 + 1, j] = np.arange(n, n + 2 * Nx12 + 1)
        xs.append(np.linspace(0, x_max, 2 * Nx12 + 1))
        ys.append(np.full(2 * Nx12 + 1, cy[j]))
        n += 2 * Nx12 + 1
    coord = np.vstack([np.concatenate(xs), np.concatenate(ys)])
    els = []
    for (jlo, jhi, ilen) in ((1, Ny1, Nx), (Ny1 + 1, Ny, Nx12)):
        for j in range(jlo, jhi + 1):
            for i in range(1, ilen + 1):
                a, b = 2 * i - 2, 2 * j - 2   # 0-based (2i-1, 2j-1)
                els.append([C[a, b], C[a + 2, b], C[a, b + 2], C[a + 1, b + 1], C[a, b + 1], C[a + 1, b]])
                els.append([C[a + 2, b + 2], C[a, b + 2], C[a + 2, b], C[a + 1, b + 1], C[a + 2, b + 1], C[a + 1, b + 2]])
    elem = np.array(els, np.int32).T.copy()
    x, y = coord
    x_max = x.max() - 1e-9
    Q = np.zeros((2, coord.shape[1]), bool)
    Q[0] = (x > 0) & (y > 0) & (x < x_max)
    Q[1] = y > 0
    return Mesh(coord, elem, Q, dict(kind="slope2d", h=h, dims=(x1, x2, x3, y1, y2)))


# ----------------------------------------------------------------- geometry


def geometry_3d(mesh: Mesh, dhat1, dhat2, dhat3, wf):
    """Physical gradients and weights, elastic_stiffness_matrix_3D.m:49-96,148.
    Returns DPhi1, DPhi2, DPhi3 (n_int, n_p) and WEIGHT (n_int,)."""
    X = mesh.coord[:, mesh.elem]               # (3, n_p, n_e)
    # J_ab = sum_i X_b[i] * dhat_a[i, q]   -> (n_e, n_q)
    def jac(a, b):
        return np.einsum("ie,iq->eq", X[b], (dhat1, dhat2, dhat3)[a])
    J = [[jac(a, b) for b in range(3)] for a in range(3)]
    J11, J12, J13 = J[0]
    J21, J22, J23 = J[1]
    J31, J32, J33 = J[2]
    det = J11 * (J22 * J33 - J32 * J23) - J12 * (J21 * J33 - J23 * J31) + J13 * (J21 * J32 - J22 * J31)
    inv = [[(J22 * J33 - J23 * J32) / det, -(J12 * J33 - J13 * J32) / det, (J12 * J23 - J13 * J22) / det],
           [-(J21 * J33 - J23 * J31) / det, (J11 * J33 - J13 * J31) / det, -(J11 * J23 - J13 * J21) / det],
           [(J21 * J32 - J22 * J31) / det, -(J11 * J32 - J12 * J31) / det, (J11 * J22 - J12 * J21) / det]]
    dh = (dhat1, dhat2, dhat3)
    out = []
    for r in range(3):
        d = (inv[r][0][:, :, None] * dh[0].T[None] + inv[r][1][:, :, None] * dh[1].T[None]
             + inv[r][2][:, :, None] * dh[2].T[None])          # (n_e, n_q, n_p)
        out.append(np.ascontiguousarray(d.reshape(-1, d.shape[2])))
    weight = (np.abs(det) * wf[None, :]).ravel()
    return out[0], out[1], out[2], weight


def geometry_2d(mesh: Mesh, dhat1, dhat2, wf):
    """Physical gradients and weights, elastic_stiffness_matrix_2D.m."""
    X = mesh.coord[:, mesh.elem]
    J11 = np.einsum("ie,iq->eq", X[0], dhat1)
    J12 = np.einsum("ie,iq->eq", X[1], dhat1)
    J21 = np.einsum("ie,iq->eq", X[0], dhat2)
    J22 = np.einsum("ie,iq->eq", X[1], dhat2)
    det = J11 * J22 - J12 * J21
    i11, i12, i21, i22 = J22 / det, -J12 / det, -J21 / det, J11 / det
    d1 = i11[:, :, None] * dhat1.T[None] + i12[:, :, None] * dhat2.T[None]
    d2 = i21[:, :, None] * dhat1.T[None] + i22[:, :, None] * dhat2.T[None]
    weight = (np.abs(det) * wf[None, :]).ravel()
    n_p = dhat1.shape[0]
    return (np.ascontiguousarray(d1.reshape(-1, n_p)), np.ascontiguousarray(d2.reshape(-1, n_p)), weight)


# ----------------------------------------------------------------- materials


def materials(mat_id_per_elem, n_q, mat_table, saturation=None):
    """Per-point material fields, heterogenous_materials.m:51-86.
    mat_table rows: (c0, phi_deg, psi_deg, young, poisson, gamma_sat, gamma_unsat).
    Returns dict of flat (n_int,) arrays c0, phi, psi (radians), shear, bulk, lame, gamma."""
    tab = np.asarray(mat_table, dtype=np.float64).reshape(-1, 7)
    m = np.asarray(mat_id_per_elem, np.int64)
    row = tab[m]
    c0 = row[:, 0]
    phi = row[:, 1] * np.pi / 180
    psi = row[:, 2] * np.pi / 180
    young, nu = row[:, 3], row[:, 4]
    shear = young / (2 * (1 + nu))
    bulk = young / (3 * (1 - 2 * nu))
    lame = bulk - 2 * shear / 3
    rep = lambda a: np.repeat(a, n_q)
    n_int = m.size * n_q
    sat = np.ones(n_int, bool) if saturation is None else np.asarray(saturation, bool)
    gamma = np.where(sat, rep(row[:, 5]), rep(row[:, 6]))
    return dict(c0=rep(c0), phi=rep(phi), psi=rep(psi), shear=rep(shear), bulk=rep(bulk),
                lame=rep(lame), gamma=gamma)


def elastic_fields_from_point_draws(c0, phi_deg, young, nu):
    """Per-point c0 / phi / psi=0 / moduli for point-wise material draws (the box microbenchmark)."""
    shear = young / (2 * (1 + nu))
    bulk = young / (3 * (1 - 2 * nu))
    lame = bulk - 2 * shear / 3
    n = np.size(c0)
    bc = lambda a: np.broadcast_to(np.asarray(a, np.float64), (n,)).copy()
    return dict(c0=bc(c0), phi=bc(phi_deg) * np.pi / 180, psi=np.zeros(n), shear=bc(shear),
                bulk=bc(bulk), lame=bc(lame))


def gravity_load(mesh: Mesh, hat, weight, gamma):
    """Body-force vector f_V (dim, n_n) for f_V_int = [0; -gamma; 0], vector_volume_3D.m."""
    n_q = hat.shape[1]
    n_e = mesh.n_e
    w = (weight * gamma).reshape(n_e, n_q)                  # (n_e, n_q)
    contrib = np.einsum("iq,eq->ie", hat, w)                # (n_p, n_e)
    f = np.zeros((mesh.dim, mesh.n_n))
    np.add.at(f[1], mesh.elem.ravel(), -contrib.ravel())
    return f


def davis_reduction(c0, phi, psi, lam, davis="B"):
    """Host restatement of +CONSTITUTIVE_PROBLEM/reduction.m:25-58 (used for set-up and
    checks; the device path fuses it into the constitutive kernel)."""
    c0, phi, psi = map(np.asarray, (c0, phi, psi))
    if davis == "A":
        beta = np.cos(phi) * np.cos(psi) / (1 - np.sin(phi) * np.sin(psi))
        c_l = beta * c0 / lam
        phi_l = np.arctan(beta * np.tan(phi) / lam)
    elif davis == "B":
        c1 = c0 / lam
        f1 = np.arctan(np.tan(phi) / lam)
        s1 = np.arctan(np.tan(psi) / lam)
        beta = np.cos(f1) * np.cos(s1) / (1 - np.sin(f1) * np.sin(s1))
        c_l = beta * c1
        phi_l = np.arctan(beta * np.tan(f1))
    elif davis == "C":
        c1 = c0 / lam
        f1 = np.arctan(np.tan(phi) / lam)
        beta = np.where(f1 > psi, np.cos(f1) * np.cos(psi) / (1 - np.sin(f1) * np.sin(psi)), 1.0)
        c_l = beta * c1
        phi_l = np.arctan(beta * np.tan(f1))
    else:
        raise ValueError("Davis type must be 'A', 'B' or 'C'")
    return 2 * c_l * np.cos(phi_l), np.sin(phi_l)


# ----------------------------------------------------------------- random fields


def _embedding_eigenvalues(shape, spacing, corr_len):
    """Eigenvalues of the block-circulant embedding of the exponential covariance
    exp(-r / corr_len) on a periodic grid of ``shape`` points with ``spacing`` (the
    covariance evaluated at the periodic lag min(k, m - k) * spacing per axis)."""
    lags = [np.minimum(np.arange(m), m - np.arange(m)) * d for m, d in zip(shape, spacing)]
    r2 = np.zeros(shape)
    for ax, lag in enumerate(lags):
        sh = [1] * len(shape)
        sh[ax] = -1
        r2 = r2 + (lag ** 2).reshape(sh)
    cov = np.exp(-np.sqrt(r2) / corr_len)
    return np.fft.fftn(cov).real


def gaussian_fields_circulant(lower, upper, spacing, corr_len, seed, n_fields=2, max_pad=64):
    """Independent standard Gaussian random fields with the isotropic exponential covariance
    exp(-|x - y| / corr_len), sampled on the regular grid lower + spacing * k covering the box
    [lower, upper], by circulant embedding (Dietrich & Newsam 1997, SIAM J. Sci. Comput.
    18(4):1088-1107; Wood & Chan 1994): the covariance on a periodic grid of at least twice the
    box is diagonalised by the FFT, white noise is coloured by the square roots of its
    eigenvalues, and one complex FFT gives two independent fields (real and imaginary parts).
    The periodic grid is padded until every eigenvalue is non-negative (up to ``max_pad``
    points per axis); any negative remainder is set to zero and its share reported.

    Returns (fields (n_fields, *grid_shape), grid axes, info)."""
    lower = np.asarray(lower, np.float64)
    upper = np.asarray(upper, np.float64)
    n = np.maximum(np.ceil((upper - lower) / spacing).astype(int) + 1, 2)
    axes = [lower[i] + spacing * np.arange(n[i]) for i in range(n.size)]
    pad = 0
    while True:
        m = tuple(int(2 * (k - 1) + 2 * pad) for k in n)
        lam = _embedding_eigenvalues(m, [spacing] * n.size, corr_len)
        if lam.min() >= -1e-12 * lam.max() or pad >= max_pad:
            break
        pad = max(2 * pad, 4)
    neg = float(-lam[lam < 0].sum() / lam.sum()) if (lam < 0).any() else 0.0
    sq = np.sqrt(np.maximum(lam, 0.0) / lam.size)
    rng = np.random.default_rng(seed)
    out = []
    for _ in range((n_fields + 1) // 2):
        xi = rng.standard_normal(m) + 1j * rng.standard_normal(m)
        y = np.fft.fftn(sq * xi)
        sl = tuple(slice(0, k) for k in n)
        out += [y.real[sl], y.imag[sl]]
    info = dict(grid=tuple(int(k) for k in n), embedding=m, pad=pad, negative_eigen_share=neg,
                method="circulant embedding, exponential covariance")
    return np.stack(out[:n_fields]), axes, info


def trilinear(field, axes, pts):
    """Trilinear interpolation of a grid ``field`` (nx, ny, nz) on ``axes`` at ``pts`` (3, n)."""
    idx, frac = [], []
    for a, p in zip(axes, pts):
        h = a[1] - a[0]
        t = np.clip((p - a[0]) / h, 0.0, a.size - 1 - 1e-12)
        i = np.floor(t).astype(np.int64)
        idx.append(i)
        frac.append(t - i)
    (i, j, k), (u, v, w) = idx, frac
    out = np.zeros(pts.shape[1])
    for di, wi in ((0, 1 - u), (1, u)):
        for dj, wj in ((0, 1 - v), (1, v)):
            for dk, wk in ((0, 1 - w), (1, w)):
                out += wi * wj * wk * field[i + di, j + dj, k + dk]
    return out


def lognormal_from_gaussian(g, mean, cov):
    """Lognormal values of the given mean and coefficient of variation from standard normal g."""
    s2 = np.log1p(cov ** 2)
    return np.exp(np.log(mean) - s2 / 2 + np.sqrt(s2) * g)


def integration_points(mesh: Mesh, hat):
    """Physical coordinates (dim, n_e * n_q) of the integration points, element-major
    (the point order of the per-point fields)."""
    X = mesh.coord[:, mesh.elem]                      # (dim, n_p, n_e)
    return np.einsum("dpe,pq->deq", X, hat).reshape(mesh.dim, -1)


def vector_volume(mesh: Mesh, hat, weight, f_int):
    """Load vector (dim, n_n) of a body force given per integration point, f_int (dim, n_int):
    f_V(d, node) = sum over the node's elements and their points of w * HatP * f_int(d)
    (vector_volume_3D.m / vector_volume_2D.m)."""
    n_q = hat.shape[1]
    n_e = mesh.n_e
    f_int = np.asarray(f_int, np.float64).reshape(mesh.dim, n_e, n_q)
    out = np.zeros((mesh.dim, mesh.n_n))
    w = np.asarray(weight, np.float64).reshape(n_e, n_q)
    for d in range(mesh.dim):
        contrib = np.einsum("iq,eq->ie", hat, w * f_int[d])          # (n_p, n_e)
        np.add.at(out[d], mesh.elem.ravel(), contrib.ravel())
    return out


def midpoints_p2_2d(coord, elem):
    """P1 -> P2 for triangles in the numbering of +MESH/midpoints_P2.m: the midpoint of every
    edge is numbered at its first occurrence when the elements are visited in order and, in
    each, the edges V2-V3, V3-V1, V1-V2; elem_mid rows are those three edges.  ``surf`` lists
    the boundary edges in the same order as columns [V3; V2; mid] -- V3 and V2 of the element
    the edge belongs to, for every one of its three edges (the reference's list keeps these
    two vertices whichever edge it is).  coord (2, n_n), elem (3, n_e) 0-based.  Returns
    coord_mid (2, n_mid), elem_mid (3, n_e), surf (3, n_s), all ids 0-based."""
    coord = np.asarray(coord, np.float64)
    elem = np.asarray(elem, np.int64)
    n_n, n_e = coord.shape[1], elem.shape[1]
    a = np.stack([elem[1], elem[2], elem[0]], 1)          # first vertex of edges 1, 2, 3
    b = np.stack([elem[2], elem[0], elem[1]], 1)          # second vertex
    lo, hi = np.minimum(a, b).ravel(), np.maximum(a, b).ravel()   # occurrence order: element, edge
    key = lo * n_n + hi
    uniq, first, inv, cnt = np.unique(key, return_index=True, return_inverse=True, return_counts=True)
    order = np.argsort(first, kind="stable")               # edges by first occurrence
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    mid_of_occ = rank[inv]                                 # midpoint number of every occurrence
    elem_mid = (n_n + mid_of_occ).reshape(n_e, 3).T.copy()
    fo = first[order]                                      # first occurrence of midpoint m
    coord_mid = (coord[:, lo[fo]] + coord[:, hi[fo]]) / 2
    bnd = order[cnt[order] == 1]                           # boundary edges in midpoint order
    occ = first[bnd]
    e_of = occ // 3
    surf = np.vstack([elem[2, e_of], elem[1, e_of], n_n + rank[bnd]])
    return coord_mid, elem_mid, surf


def mesh_p2_from_p1_2d(coord_p1, elem_p1):
    """(coord, elem, surf) of the P2 mesh built from a P1 triangulation by midpoints_p2_2d."""
    cm, em, surf = midpoints_p2_2d(coord_p1, elem_p1)
    return np.hstack([np.asarray(coord_p1, np.float64), cm]), np.vstack([np.asarray(elem_p1, np.int64), em]), surf

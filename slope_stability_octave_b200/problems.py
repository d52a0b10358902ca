"""Problem set-up for the benchmark workloads (host inputs + device objects).

slope_2d                2D homogeneous slope, P2 triangles, h = 0.5 (slope_stability_2D_homo_SSR.m:30-48)
slope_3d                3D homogeneous slope, P2 tets: the 2D profile extruded 40 m, mesh_P2_3D(N_h = 1,
                        15, 10, 15, 10, 10, 40) (slope_stability_3D_homo_SSR.m parameters)
slope_3d_layered        3D slope with horizontal material layers (heterogeneous), see
                        ``layered_material_ids``
slope_3d_random_field   3D slope with lognormal random-field strength (limit-load workload)``
slope_3d_from_mesh      a P2 tetrahedral mesh given as arrays (e.g. one of the reference's HDF5
                        meshes read by h5mesh.load_mesh_P2), homogeneous or with per-element
                        material ids (slope_stability_3D_{homo,hetero}_SSR.m)

Material rows are (c0 [kPa], phi [deg], psi [deg], E [kPa], nu, gamma_sat, gamma_unsat).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import fem
from .constitutive import CONSTITUTIVE
from .device import DeviceMesh
from .linear_solvers import set_linear_solver

HOMO = [6.0, 45.0, 0.0, 40000.0, 0.3, 20.0, 20.0]

# continuation parameters of the reference drivers
# the stored runs of slope_stability_3D_hetero_SSR.m (mesh SSR_hetero_ada_L1.h5): material
# rows by the mesh's material id 0..3 (cover layer, general foundation, relatively weak
# foundation, general slope mass) and the script's continuation parameters
HETERO_SSR_MATERIALS = [[15.0, 30.0, 0.0, 10000.0, 0.33, 19.0, 19.0],
                        [15.0, 38.0, 0.0, 50000.0, 0.30, 22.0, 22.0],
                        [10.0, 35.0, 0.0, 50000.0, 0.30, 21.0, 21.0],
                        [18.0, 32.0, 0.0, 20000.0, 0.33, 20.0, 20.0]]
SSR_3D = dict(lambda_init=0.9, d_lambda_init=0.1, d_lambda_min=1e-3, d_lambda_diff_scaled_min=1e-3,
              step_max=100, omega_max_stop=3000.0, it_newt_max=100, it_damp_max=10, tol=1e-4, r_min=1e-4)
SSR_2D = dict(lambda_init=0.9, d_lambda_init=0.05, d_lambda_min=1e-5, d_lambda_diff_scaled_min=1e-3,
              step_max=100, omega_max_stop=5e3, it_newt_max=30, it_damp_max=10, tol=1e-4, r_min=1e-4)
# omega = f(Q)'U(Q) grows with the loaded volume; for the 40 m deep extruded slope the
# reference 3D driver's omega_max_stop = 3000 (chosen for its own smaller mesh) would stop at
# once, so the bound is lifted to the 2D script's 7e7 and the lambda-increment test stops.
SSR_3D_EXTRUDED = dict(SSR_3D, omega_max_stop=7e7)
SSR_3D_HETERO = dict(SSR_3D, lambda_init=1.0, omega_max_stop=1.2e7, it_newt_max=200)
# limit-load continuation parameters of slope_stability_3D_homo_LL.m:82-96 and
# slope_stability_2D_homo_LL.m:154-163
LL_3D = dict(d_t_min=1e-3, step_max=100, omega_max=5100.0, it_newt_max=200, it_damp_max=10, tol=1e-4, r_min=1e-4)
# the 40 m deep extruded slope carries ~40x the work f'U of the reference's 1 m-thick LL
# mesh scale, so its omega bound is lifted as for SSR; runs stop on the t increment or a
# step budget
LL_3D_EXTRUDED = dict(LL_3D, omega_max=7e7)
LL_2D = dict(d_t_min=1e-3, step_max=100, omega_max=2000.0, it_newt_max=100, it_damp_max=10, tol=1e-4, r_min=1e-4)


@dataclass
class Problem:
    mesh: fem.Mesh
    dphi: tuple
    weight: np.ndarray
    hat: np.ndarray
    n_q: int
    mat: dict
    f: np.ndarray           # (dim, n_n)
    Davis_type: str = "B"
    dmesh: DeviceMesh = None
    cons: CONSTITUTIVE = None

    @property
    def dim(self):
        return self.mesh.dim

    def to_device(self):
        self.dmesh = DeviceMesh(self.mesh, self.dphi, self.weight, self.n_q)
        m = self.mat
        self.cons = CONSTITUTIVE(self.dmesh, m["c0"], m["phi"], m["psi"], self.Davis_type, m["shear"], m["bulk"],
                                 m["lame"])
        return self

    def f_device(self):
        return torch.from_numpy(np.ascontiguousarray(self.f.T).ravel()).to(self.dmesh.device)

    def solver(self, solver_type="DFGMRES_B200", tol=1e-1, maxit=100, defl_tol=1e-3, amg_opts=None):
        return set_linear_solver(solver_type, tol, maxit, defl_tol, 0, self.dmesh, self.mesh.coord, amg_opts)


def _assemble_problem(mesh, mat_ids, table, davis="B"):
    if mesh.dim == 3:
        xi, wf = fem.quadrature_p2_tet()
        hat, d1, d2, d3 = fem.local_basis_p2_tet(xi)
        D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
        dphi = (D1, D2, D3)
    else:
        xi, wf = fem.quadrature_p2_tri()
        hat, d1, d2 = fem.local_basis_p2_tri(xi)
        D1, D2, W = fem.geometry_2d(mesh, d1, d2, wf)
        dphi = (D1, D2)
    n_q = wf.size
    mat = fem.materials(mat_ids, n_q, table)
    f = fem.gravity_load(mesh, hat, W, mat["gamma"])
    return Problem(mesh, dphi, W, hat, n_q, mat, f, davis)


def slope_2d(h=0.5, mat=HOMO):
    x1, x3, y1, y2 = 15.0, 15.0, 10.0, 10.0
    x2 = y2 / np.tan(45 * np.pi / 180)
    mesh = fem.mesh_p2_2d(h, x1, x2, x3, y1, y2)
    return _assemble_problem(mesh, np.zeros(mesh.n_e, int), mat)


def slope_3d(N_h=1, dims=(15, 10, 15, 10, 10, 40), mat=HOMO):
    mesh = fem.mesh_p2_3d(N_h, *dims)
    return _assemble_problem(mesh, np.zeros(mesh.n_e, int), mat)


def slope_3d_from_mesh(coord, elem, Q, material=None, table=HOMO):
    """Problem on a given P2 tetrahedral mesh: coord (3, n_n), elem (10, n_e) 0-based, Q (3, n_n)
    free-DOF mask; ``material`` = per-element row index into ``table`` (None: all row 0)."""
    mesh = fem.Mesh(np.ascontiguousarray(coord, np.float64), np.ascontiguousarray(elem, np.int64),
                    np.ascontiguousarray(Q, bool))
    ids = np.zeros(mesh.n_e, int) if material is None else np.asarray(material, int)
    return _assemble_problem(mesh, ids, table)


# four horizontal layers, thicknesses 5/5/10/20 m measured from the crest (y = 20 m)
# downward and clipped at the base (y = 0): the body is 20 m high, so the two lower layers
# of the listed four fall below the base and only the first three (plus the clipped 10 m one)
# carry material.  Rows: (c0, phi, psi, E, nu, gamma, gamma).
SLOPE_LAYERS = [[15.0, 30.0, 0.0, 50000.0, 0.30, 19.0, 19.0],
               [10.0, 35.0, 0.0, 40000.0, 0.30, 20.0, 20.0],
               [18.0, 25.0, 0.0, 60000.0, 0.30, 21.0, 21.0],
               [6.0, 45.0, 0.0, 40000.0, 0.30, 20.0, 20.0]]
SLOPE_LAYER_THICKNESS = (5.0, 5.0, 10.0, 20.0)


def layered_material_ids(mesh, top=20.0, thickness=SLOPE_LAYER_THICKNESS):
    """Layer index of every element by the depth of its centroid below ``top``."""
    yc = mesh.coord[1, mesh.elem[:4]].mean(axis=0)
    depth = top - yc
    bounds = np.cumsum(thickness)
    return np.minimum(np.searchsorted(bounds, depth, side="right"), len(thickness) - 1)


def slope_3d_layered(N_h=1, dims=(15, 10, 15, 10, 10, 40)):
    mesh = fem.mesh_p2_3d(N_h, *dims)
    ids = layered_material_ids(mesh, top=dims[3] + dims[4])
    return _assemble_problem(mesh, ids, SLOPE_LAYERS)


# strength random field of the limit-load workload: lognormal c and phi, independent,
# isotropic exponential correlation; E = 40 MPa, nu = 0.3, gamma = 20 kN/m^3 everywhere
RANDOM_FIELD_STRENGTH = dict(c_mean=10.0, c_cov=0.3, phi_mean=35.0, phi_cov=0.1, corr_len=5.0, young=40000.0, nu=0.3,
                         gamma=20.0, spacing=0.5)


def random_field_materials(mesh, hat, seed, rf=RANDOM_FIELD_STRENGTH):
    """Per-integration-point material of a slope whose cohesion and friction angle are
    independent lognormal random fields (means and coefficients of variation in ``rf``) with
    the exponential correlation exp(-r / corr_len).  The two standard Gaussian fields come
    from one circulant-embedding draw on a grid of ``spacing`` over the mesh's bounding box
    (fem.gaussian_fields_circulant) and are interpolated trilinearly to the integration
    points.  The reference scripts have no random fields; this generator is this library's."""
    lo, hi = mesh.coord.min(axis=1), mesh.coord.max(axis=1)
    G, axes, info = fem.gaussian_fields_circulant(lo, hi, rf["spacing"], rf["corr_len"], seed, n_fields=2)
    X = fem.integration_points(mesh, hat)
    g_c = fem.trilinear(G[0], axes, X)
    g_phi = fem.trilinear(G[1], axes, X)
    c0 = fem.lognormal_from_gaussian(g_c, rf["c_mean"], rf["c_cov"])
    phi = fem.lognormal_from_gaussian(g_phi, rf["phi_mean"], rf["phi_cov"])
    mat = fem.elastic_fields_from_point_draws(c0, phi, rf["young"], rf["nu"])
    mat["gamma"] = np.full(c0.size, rf["gamma"])
    return mat, info


def slope_3d_random_field(N_h=1, dims=(15, 10, 15, 10, 10, 40), seed=20261203, rf=RANDOM_FIELD_STRENGTH):
    """The extruded 3D slope with lognormal random-field strength (limit-load workload)."""
    mesh = fem.mesh_p2_3d(N_h, *dims)
    xi, wf = fem.quadrature_p2_tet()
    hat, d1, d2, d3 = fem.local_basis_p2_tet(xi)
    D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
    mat, info = random_field_materials(mesh, hat, seed, rf)
    f = fem.gravity_load(mesh, hat, W, mat["gamma"])
    P = Problem(mesh, (D1, D2, D3), W, hat, wf.size, mat, f, "B")
    mesh.info["random_field"] = info
    return P

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
slope_3d_seepage        the 3D homogeneous slope with a phreatic surface: seepage on the GPU,
                        then saturated unit weights and pore-pressure forces in the load
                        (slope_stability_3D_homo_seepage_SSR.m)
franz_dam               the 2D Franz dam of slope_stability_2D_Franz_dam_SSR.m (P1 mesh arrays of
                        meshes/Franz_dam, ten material zones, seepage on the GPU)

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
        if self.dmesh is None:
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


# ----------------------------------------------------------------- seepage-coupled problems


def seepage_coupled(mesh, mat_ids, table, hat, dphi, W, n_q, Q_w, pw_D, conduct0, solver_opts=None, davis="B",
                    log=None):
    """Problem whose load carries the pore pressure of an unconfined seepage solution:
    the seepage problem runs on the device (seepage.seepage_problem), its element saturation
    selects gamma_sat / gamma_unsat per point (heterogenous_materials.m:84-86) and the body
    force is f_V_int = [-grad_p(1); -grad_p(2) - gamma; -grad_p(3)] (the seepage scripts'
    f_V_int, integrated by vector_volume).  The device mesh is kept for the mechanics."""
    from . import seepage
    dmesh = DeviceMesh(mesh, dphi, W, n_q)
    o = dict(tolerance=1e-6, max_iterations=200, deflation_tolerance=1e-3)
    o.update(solver_opts or {})
    solver = seepage.seepage_solver(dmesh, Q_w, **o)
    pw, grad_p, sat, stats = seepage.seepage_problem(dmesh, hat, Q_w, pw_D, conduct0, solver=solver, log=log)
    sat_e = sat.cpu().numpy()
    saturation = np.repeat(sat_e, n_q)
    mat = fem.materials(mat_ids, n_q, table, saturation=saturation)
    gp = grad_p.cpu().numpy().T                                    # (dim, n_int)
    f_int = -gp
    f_int[1] -= mat["gamma"]
    f = fem.vector_volume(mesh, hat, W, f_int)
    P = Problem(mesh, dphi, W, hat, n_q, mat, f, davis, dmesh=dmesh)
    P.seepage = dict(pw=pw, grad_p=grad_p, mater_sat=sat, stats=stats, Q_w=Q_w, pw_D=pw_D)
    return P


SEEPAGE_HOMO = dict(k=1.0, y21=2.0, y22=6.0)


def homo_slope_seepage_bc(coord, x1=15.0, x2=10.0, x3=15.0, y1=10.0, y2=10.0, y21=2.0, y22=6.0, grho=9.81):
    """Q_w and pw_D of slope_stability_3D_homo_seepage_SSR.m:108-133: the pressure head of a
    phreatic line y21 above the toe level at the slope face and y22 higher at x = 0."""
    x, y = coord[0], coord[1]
    Q_w = np.ones(coord.shape[1], bool)
    Q_w[x <= 0.001] = False
    Q_w[x >= x1 + x2 + x3 - 0.001] = False
    Q_w[y >= y1 + y2 - 0.001] = False
    Q_w[(y >= y1 - 0.001) & (x >= x1 + x2 - 0.001)] = False
    Q_w[(y >= y1 - 0.001) & (y >= -(y2 / x2) * x + y1 + y2 * (1 + x1 / x2) - 0.001)] = False
    pw_D = np.zeros(coord.shape[1])
    x_bar = x1 + (1 - y21 / y2) * x2
    left = (x < x_bar) & (y <= -(y22 / x_bar) * x + y1 + y21 + y22)
    right = x >= x_bar
    pw_D[left] = grho * ((y22 / x_bar) * (x_bar - x[left]) + y1 + y21 - y[left])
    pw_D[right] = grho * (y1 + y21 - y[right])
    return Q_w, pw_D


def slope_3d_seepage(N_h=1, dims=(15, 10, 15, 10, 10, 5), mat=HOMO, solver_opts=None, log=None):
    """The 3D homogeneous slope of slope_stability_3D_homo_seepage_SSR.m (z = 5 m, k = 1)."""
    mesh = fem.mesh_p2_3d(N_h, *dims)
    xi, wf = fem.quadrature_p2_tet()
    hat, d1, d2, d3 = fem.local_basis_p2_tet(xi)
    D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
    x1, x2, x3, y1, y2, _ = dims
    Q_w, pw_D = homo_slope_seepage_bc(mesh.coord, x1, x2, x3, y1, y2, SEEPAGE_HOMO["y21"], SEEPAGE_HOMO["y22"])
    conduct0 = np.full(mesh.n_e * wf.size, SEEPAGE_HOMO["k"])
    return seepage_coupled(mesh, np.zeros(mesh.n_e, int), mat, hat, (D1, D2, D3), W, wf.size, Q_w, pw_D, conduct0,
                           solver_opts, log=log)


# slope_stability_2D_Franz_dam_SSR.m:30-64: ten zones (c0, phi, psi, E, nu, gamma_sat,
# gamma_unsat) and their conductivities
FRANZ_DAM_MATERIALS = [[50.0, 42.0, 42.0, 16000.0, 0.4, 27.0, 27.0],
                       [0.5, 41.0, 0.0, 16000.0, 0.4, 22.0, 22.0],
                       [0.5, 40.0, 0.0, 16000.0, 0.4, 23.0, 23.0],
                       [0.0, 38.0, 0.0, 16000.0, 0.4, 23.0, 23.0],
                       [10.0, 25.0, 0.0, 16000.0, 0.4, 22.0, 22.0],
                       [0.5, 41.0, 0.0, 16000.0, 0.4, 22.0, 22.0],
                       [75.0, 42.0, 42.0, 16000.0, 0.4, 27.0, 27.0],
                       [0.0, 38.0, 0.0, 16000.0, 0.4, 23.0, 23.0],
                       [0.5, 41.0, 0.0, 16000.0, 0.4, 23.0, 23.0],
                       [0.5, 41.0, 0.0, 16000.0, 0.4, 21.0, 21.0]]
FRANZ_DAM_K = [1.0e-5, 1.0e-4, 5.0e-5, 5.0e-6, 1.0e-9, 1.0e-4, 2.0e-9, 5.0e-6, 5.0e-5, 5.0e-4]
# continuation parameters of the same script (:151-162)
SSR_FRANZ_DAM = dict(lambda_init=0.7, d_lambda_init=0.05, d_lambda_min=1e-5, d_lambda_diff_scaled_min=0.01,
                     step_max=100, omega_max_stop=1e10, it_newt_max=30, it_damp_max=10, tol=1e-5, r_min=1e-4)


def franz_dam_seepage_bc(coord, surf, grho=9.81):
    """Q_w and pw_D of slope_stability_2D_Franz_dam_SSR.m:100-128: the boundary edges whose
    (first two listed) vertices lie above y = -399.9 are Dirichlet for the pressure, which
    follows the upstream and downstream water levels (piecewise linear between x1 and x2)."""
    Q_D = (coord[1, surf[0]] + coord[1, surf[1]]) / 2 >= -400 + 1e-1
    Q_w = np.ones(coord.shape[1], bool)
    Q_w[np.unique(surf[:, Q_D])] = False
    x1, y1, x2, y2 = -82.5, -50.0, 172.5, -112.0
    x, y = coord
    pw_D = np.zeros(coord.shape[1])
    up = (x < x1 + 1e-9) & (y < y1)
    mid = (x >= x1 + 1e-9) & (x < x2 + 1e-9) & (y < ((y2 - y1) / (x2 - x1)) * (x - x1) + y1)
    down = (x >= x2 + 1e-9) & (y < y2)
    pw_D[up] = grho * (y1 - y[up])
    pw_D[mid] = grho * (((y2 - y1) / (x2 - x1)) * (x[mid] - x1) + y1 - y[mid])
    pw_D[down] = grho * (y2 - y[down])
    return Q_w, pw_D


def franz_dam(coords_p1, elems_p1, materials_1based, solver_opts=None, log=None):
    """The 2D Franz dam (load_mesh_Franz_dam.m with 'P2', the script's seepage and
    materials).  coords_p1 (n, 2), elems_p1 (n_e, 3) 0-based, materials_1based (n_e,): the
    arrays of meshes/Franz_dam/{coordinates,elements,materials}.txt."""
    coord, elem, surf = fem.mesh_p2_from_p1_2d(np.asarray(coords_p1, np.float64).T, np.asarray(elems_p1).T)
    mater = np.asarray(materials_1based, np.int64).reshape(-1) - 1
    x_max, x_min, y_min = coord[0].max(), coord[0].min(), coord[1].min()
    Q = np.zeros((2, coord.shape[1]), bool)
    Q[0] = (coord[0] > x_min + 0.2) & (coord[1] > y_min + 0.2) & (coord[0] < x_max - 0.2)
    Q[1] = coord[1] > y_min + 0.2
    mesh = fem.Mesh(coord, elem, Q, dict(kind="franz_dam"))
    xi, wf = fem.quadrature_p2_tri()
    hat, d1, d2 = fem.local_basis_p2_tri(xi)
    D1, D2, W = fem.geometry_2d(mesh, d1, d2, wf)
    Q_w, pw_D = franz_dam_seepage_bc(coord, surf)
    conduct0 = np.repeat(np.asarray(FRANZ_DAM_K)[mater], wf.size)
    return seepage_coupled(mesh, mater, FRANZ_DAM_MATERIALS, hat, (D1, D2), W, wf.size, Q_w, pw_D, conduct0,
                           solver_opts, log=log)

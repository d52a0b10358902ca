"""Generate seepage_oracle.npz: the reference's Franz dam mesh, the stored run of its notebook,
and the oracle's seepage and seepage-coupled SSR results.

    python tests/golden/make_seepage_fixtures.py

Reads (in this container only) the reference's meshes/Franz_dam/{coordinates, elements,
materials}.txt and the printed outputs of slope_stability_2D_Franz_dam_SSR.ipynb, and stores:

  franz_coord_p1, franz_elem_p1 (0-based), franz_mat (1-based)   the mesh arrays
  stored_seepage_newton                       seepage Newton iterations of the stored run
  stored_direct_omega_init, stored_direct_lambda, stored_indirect_lambda, stored_indirect_omega_init
                                              the accepted steps printed by the stored run
  franz_pw, franz_sat, franz_newton          oracle seepage (oracle/seepage_ref.py, direct solves)
  franz_lambda, franz_omega, franz_its        oracle SSR indirect continuation (init + 3 steps) on
                                              the seepage-coupled load, direct solves
  homo3d_pw, homo3d_sat, homo3d_newton        oracle seepage of slope_stability_3D_homo_seepage_SSR.m's
                                              set-up on mesh_P2_3D(1, 15, 10, 15, 10, 10, z = 1)
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import seepage_ref as sr  # noqa: E402
from oracle.drivers import DirectSolver, OracleConstitutive, SSR_indirect_continuation  # noqa: E402
from slope_stability_octave_b200 import fem, problems  # noqa: E402

REF = "/root/reference/slope_stability"


def stored_run():
    nb = json.load(open(os.path.join(REF, "slope_stability_2D_Franz_dam_SSR.ipynb")))
    text = "\n".join("".join(o.get("text", "")) for c in nb["cells"] if c["cell_type"] == "code"
                     for o in c.get("outputs", []))
    direct, indirect = text.split("Indirect continuation method")
    seep = int(re.search(r"seepage_newton summary: status=converged, it=(\d+)", text).group(1))
    om_d = float(re.search(r"omega_init = ([0-9.]+)", direct).group(1))
    om_i = float(re.search(r"omega_init = ([0-9.]+)", indirect).group(1))
    lam_d = [float(x) for x in re.findall(r"accepted: lambda=([0-9.]+)", direct)]
    lam_i = [float(x) for x in re.findall(r"accepted: lambda=([0-9.]+)", indirect)]
    return dict(stored_seepage_newton=seep, stored_direct_omega_init=om_d, stored_indirect_omega_init=om_i,
                stored_direct_lambda=np.array(lam_d), stored_indirect_lambda=np.array(lam_i))


def franz_oracle(c, e, m, steps=3):
    coord, elem, Q, mater, surf = sr.franz_dam_mesh(c, e, m)
    mesh = fem.Mesh(coord, elem, Q)
    xi, wf = fem.quadrature_p2_tri()
    hat, d1, d2 = fem.local_basis_p2_tri(xi)
    D1, D2, W = fem.geometry_2d(mesh, d1, d2, wf)
    Q_w, pw_D = sr.franz_dam_seepage_bc(coord, surf)
    conduct = np.repeat(np.asarray(problems.FRANZ_DAM_K)[mater], wf.size)
    pw, grad_p, sat, st = sr.seepage_problem(coord, elem, Q_w, pw_D, sr.GRHO, conduct, hat, (D1, D2), W)
    mat = fem.materials(mater, wf.size, problems.FRANZ_DAM_MATERIALS, saturation=np.repeat(sat, wf.size))
    f_int = -grad_p.T.copy()
    f_int[1] -= mat["gamma"]
    f = fem.vector_volume(mesh, hat, W, f_int)
    cons = OracleConstitutive(mesh, (D1, D2), W, wf.size, mat)
    lh, oh, its, _ = SSR_indirect_continuation(problems.SSR_FRANZ_DAM, cons.Q, np.ascontiguousarray(f.T).ravel(),
                                              cons, DirectSolver(), max_steps_after_init=steps)
    return dict(franz_pw=pw, franz_sat=sat, franz_newton=st["iterations"], franz_lambda=np.asarray(lh),
                franz_omega=np.asarray(oh), franz_its=np.asarray(its, np.int64))


def homo3d_oracle():
    mesh = fem.mesh_p2_3d(1, 15, 10, 15, 10, 10, 1)
    xi, wf = fem.quadrature_p2_tet()
    hat, d1, d2, d3 = fem.local_basis_p2_tet(xi)
    D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
    Q_w, pw_D = sr.homo_slope_seepage_bc(mesh.coord)
    pw, _, sat, st = sr.seepage_problem(mesh.coord, mesh.elem, Q_w, pw_D, sr.GRHO, np.ones(mesh.n_e * wf.size), hat,
                                        (D1, D2, D3), W)
    return dict(homo3d_pw=pw, homo3d_sat=sat, homo3d_newton=st["iterations"])


def main():
    d = os.path.join(REF, "meshes", "Franz_dam")
    c = np.loadtxt(os.path.join(d, "coordinates.txt"))
    e = np.loadtxt(os.path.join(d, "elements.txt")).astype(np.int64)
    m = np.loadtxt(os.path.join(d, "materials.txt")).astype(np.int64)
    out = dict(franz_coord_p1=c, franz_elem_p1=e, franz_mat=m)
    out.update(stored_run())
    out.update(franz_oracle(c, e, m))
    out.update(homo3d_oracle())
    for k, v in out.items():
        print(k, np.shape(v), v if np.size(v) < 12 else "")
    np.savez_compressed(os.path.join(HERE, "seepage_oracle.npz"), **out)


if __name__ == "__main__":
    main()

"""Generate the golden fixtures in this folder from the reference's own C kernels.

    python tests/golden/make_golden.py

Requires the reference MEX sources compiled unchanged into oracle/_ref (``make -C oracle ref``,
which reads them from the reference checkout).  The fixtures pin the oracle on machines where
the reference tree is absent.  Inputs are seeded; outputs are exactly what the reference's
constitutive_problem_{2,3}D_SDS_mex and assemble_K_tangent_vals{,_2D} return for them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import native  # noqa: E402
from oracle.octave_ref import OctavePattern  # noqa: E402
from slope_stability_octave_b200 import fem, workloads  # noqa: E402


def small_3d_mesh():
    m = fem.mesh_p2_3d(1, 2, 1, 2, 1, 1, 2)
    xi, wf = fem.quadrature_p2_tet()
    hat, a, b, c = fem.local_basis_p2_tet(xi)
    d1, d2, d3, w = fem.geometry_3d(m, a, b, c, wf)
    return m, (d1, d2, d3), w


def small_2d_mesh():
    m = fem.mesh_p2_2d(1.0, 3, 2, 3, 2, 2)
    xi, wf = fem.quadrature_p2_tri()
    hat, a, b = fem.local_basis_p2_tri(xi)
    d1, d2, w = fem.geometry_2d(m, a, b, wf)
    return m, (d1, d2), w


def main():
    if not native.ref_available():
        native.build(ref=True)
    # ---- 3D constitutive: 1000 points, 200 per branch, margins >= 1e-8
    d = workloads.constitutive_points(1000, seed=11)
    S, DS = native.ref_constitutive(3, d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"])
    np.savez_compressed(os.path.join(HERE, "constitutive_3d.npz"), E=d["E"], c_bar=d["c_bar"],
                        sin_phi=d["sin_phi"], shear=d["shear"], bulk=d["bulk"], lame=d["lame"],
                        branch=d["target"], S=S, DS=DS)
    # ---- 2D constitutive: 600 random plane strains around the yield strain
    rng = np.random.default_rng(12)
    n = 600
    mat = fem.elastic_fields_from_point_draws(rng.uniform(5, 15, n), rng.uniform(25, 45, n), 40000.0, 0.3)
    cb, sp = fem.davis_reduction(mat["c0"], mat["phi"], mat["psi"], 1.0)
    E2 = rng.normal(size=(n, 3)) * (cb / (2 * mat["shear"]))[:, None] * rng.uniform(0.1, 4, n)[:, None]
    E2[: n // 6] = np.abs(E2[: n // 6]) * [1, 1, 0.01]      # tension-dominated -> apex/right edge
    S2, DS2 = native.ref_constitutive(2, E2, cb, sp, mat["shear"], mat["bulk"], mat["lame"])
    np.savez_compressed(os.path.join(HERE, "constitutive_2d.npz"), E=E2, c_bar=cb, sin_phi=sp,
                        shear=mat["shear"], bulk=mat["bulk"], lame=mat["lame"], S=S2, DS=DS2)
    # ---- 3D assembly on a small extruded slope (96 P2 tets)
    m, dphi, w = small_3d_mesh()
    mat = fem.materials(np.zeros(m.n_e, int), 11, [6, 45, 0, 40000, 0.3, 20, 20])
    pat = OctavePattern(3, m.elem, m.n_n, dphi, w, m.Q, mat["shear"], mat["bulk"])
    pts = workloads.constitutive_points(w.size, seed=13)
    _, DS3 = native.ref_constitutive(3, pts["E"], pts["c_bar"], pts["sin_phi"], mat["shear"], mat["bulk"], mat["lame"])
    smap = pat.scatter_map()
    V = native.ref_assemble(3, dphi[0], dphi[1], dphi[2], DS3, w, smap, 11, pat.nnz)
    np.savez_compressed(os.path.join(HERE, "assembly_3d.npz"), DS=DS3, ref_I=pat.ref_I, ref_J=pat.ref_J,
                        transpose_perm=pat.transpose_perm, V_elast=pat.V_elast, scatter_map=smap, V_tang=V)
    # ---- 2D assembly on a small slope
    m2, dphi2, w2 = small_2d_mesh()
    mat2 = fem.materials(np.zeros(m2.n_e, int), 7, [6, 45, 0, 40000, 0.3, 20, 20])
    pat2 = OctavePattern(2, m2.elem, m2.n_n, dphi2, w2, m2.Q, mat2["shear"], mat2["bulk"])
    rng = np.random.default_rng(14)
    cb2, sp2 = fem.davis_reduction(mat2["c0"], mat2["phi"], mat2["psi"], 1.0)
    E22 = rng.normal(size=(w2.size, 3)) * 1e-3
    _, DS22 = native.ref_constitutive(2, E22, cb2, sp2, mat2["shear"], mat2["bulk"], mat2["lame"])
    smap2 = pat2.scatter_map()
    V2 = native.ref_assemble(2, dphi2[0], dphi2[1], None, DS22, w2, smap2, 7, pat2.nnz)
    np.savez_compressed(os.path.join(HERE, "assembly_2d.npz"), DS=DS22, ref_I=pat2.ref_I, ref_J=pat2.ref_J,
                        transpose_perm=pat2.transpose_perm, V_elast=pat2.V_elast, scatter_map=smap2, V_tang=V2)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

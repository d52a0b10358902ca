"""Generate mesh_ssr3d_stored_runs.npz: the reference's two 3D SSR meshes and its stored runs.

    python tests/golden/make_mesh_fixtures.py [reference checkout, default /root/reference]

Reads, from the reference checkout (present where the fixtures are made, not where the
tests run):

  slope_stability/meshes/SSR_homo_ada_L1.h5, SSR_hetero_ada_L1.h5
      through this library's HDF5 reader (slope_stability_octave_b200.h5mesh.load_mesh_P2,
      the arrays +MESH/load_mesh_P2.m:25-57 returns);
  slope_stability/slope_stability_3D_homo_SSR.ipynb, slope_stability_3D_hetero_SSR.ipynb
      the printed output of the reference's own runs on those meshes (HYPRE-preconditioned
      DFGMRES at tolerance 1e-1, Newton 1e-4): the mesh sizes, omega of the two init-phase
      points, then per accepted continuation step lambda, omega and the Newton iterations.

Stores for each case (homo, hetero): coord (3, n_n), elem (10, n_e, 0-based), Q (3, n_n),
material (n_e), the reference's n_nodes / n_unknowns / n_elements, omega1, omega2 and the
step histories.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from slope_stability_octave_b200.h5mesh import load_mesh_P2  # noqa: E402

CASES = {"homo": ("SSR_homo_ada_L1.h5", "slope_stability_3D_homo_SSR.ipynb"),
         "hetero": ("SSR_hetero_ada_L1.h5", "slope_stability_3D_hetero_SSR.ipynb")}


def notebook_text(path):
    nb = json.load(open(path))
    return "".join("".join(o.get("text", "")) for c in nb["cells"] for o in c.get("outputs", []))


def stored_run(text):
    m = re.search(r"number of nodes =(\d+)\s+number of unknowns =(\d+)\s+number of elements =(\d+)", text)
    om = re.search(r"omega1 = ([0-9.e+-]+), omega2 = ([0-9.e+-]+)", text)
    acc = re.findall(r"accepted: lambda=([0-9.e+-]+), .*?, omega=([0-9.e+-]+),", text)
    its = re.findall(r"newton_ind_SSR summary: status=converged, it=(\d+)", text)
    if not (m and om and acc) or len(acc) != len(its):
        raise RuntimeError("stored run not found in the notebook output")
    return dict(sizes=np.array([int(x) for x in m.groups()], np.int64),
                omega12=np.array([float(om.group(1)), float(om.group(2))]),
                lam=np.array([float(a) for a, _ in acc]), omega=np.array([float(b) for _, b in acc]),
                newton=np.array([int(x) for x in its], np.int64))


def main(ref="/root/reference"):
    out = {}
    for case, (mesh_file, nb) in CASES.items():
        coord, elem, surf, Q, material, boundary = load_mesh_P2(os.path.join(ref, "slope_stability", "meshes",
                                                                              mesh_file))
        run = stored_run(notebook_text(os.path.join(ref, "slope_stability", nb)))
        n_n, n_unk, n_e = run["sizes"]
        assert coord.shape[1] == n_n and elem.shape[1] == n_e and int(Q.sum()) == n_unk, case
        out[f"{case}_coord"] = coord
        out[f"{case}_elem"] = elem.astype(np.int32)
        out[f"{case}_Q"] = Q
        out[f"{case}_material"] = material.astype(np.int8)
        for k, v in run.items():
            out[f"{case}_{k}"] = v
        print(case, coord.shape, elem.shape, int(Q.sum()), "steps", run["lam"].size, "final lambda", run["lam"][-1])
    np.savez_compressed(os.path.join(HERE, "mesh_ssr3d_stored_runs.npz"), **out)


if __name__ == "__main__":
    main(*sys.argv[1:])

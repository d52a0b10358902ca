"""HDF5 mesh ingestion (h5mesh, +MESH/load_mesh_P2.m:25-57) against the reference's own mesh
files, where the reference checkout is present (the machine that makes the fixtures): every
HDF5 mesh of slope_stability/meshes/ reads, the two SSR meshes give the node, unknown and
element counts the reference's notebooks print, and tests/golden/mesh_ssr3d_stored_runs.npz
regenerates exactly from them."""
import glob
import os

import numpy as np
import pytest

from slope_stability_octave_b200 import h5mesh

REF = "/root/reference/slope_stability"
MESHES = os.path.join(REF, "meshes")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "mesh_ssr3d_stored_runs.npz")

needs_ref = pytest.mark.skipif(not os.path.isdir(MESHES), reason="reference checkout not present")


@needs_ref
def test_every_reference_mesh_reads():
    files = sorted(glob.glob(os.path.join(MESHES, "*.h5")))
    assert len(files) >= 10
    for fn in files:
        f = h5mesh.H5File(fn)
        keys = f.keys()
        for k in keys:
            a = f.read("/" + k)
            assert a.size > 0 and np.all(np.isfinite(a.astype(np.float64))), (fn, k)
        if {"elem", "face", "node", "boundary"} <= set(keys):
            coord, elem, surf, Q, material, boundary = h5mesh.load_mesh_P2(fn)
            assert coord.shape[0] == Q.shape[0] == 3 and coord.shape[1] == Q.shape[1]
            assert elem.min() >= 0 and elem.max() < coord.shape[1]
            assert surf.shape[1] == boundary.size and material.size == elem.shape[1]


@needs_ref
def test_ssr_meshes_match_reference_counts_and_fixture():
    g = np.load(GOLDEN)
    for case, fn, counts in (("homo", "SSR_homo_ada_L1.h5", (25591, 71947, 16615)),
                             ("hetero", "SSR_hetero_ada_L1.h5", (27605, 80362, 18419))):
        coord, elem, surf, Q, material, boundary = h5mesh.load_mesh_P2(os.path.join(MESHES, fn))
        assert (coord.shape[1], int(Q.sum()), elem.shape[1]) == counts
        assert np.array_equal(g[f"{case}_coord"], coord)
        assert np.array_equal(g[f"{case}_elem"], elem)
        assert np.array_equal(g[f"{case}_Q"], Q)
        assert np.array_equal(g[f"{case}_material"], material)
        assert tuple(g[f"{case}_sizes"]) == counts


def test_fixture_meshes_are_consistent():
    """The fixture's meshes are valid P2 tetrahedral meshes (runs without the reference)."""
    from slope_stability_octave_b200 import problems
    g = np.load(GOLDEN)
    for case in ("homo", "hetero"):
        coord, elem, Q = g[f"{case}_coord"], g[f"{case}_elem"], g[f"{case}_Q"]
        # the homogeneous script ignores the file's material ids (material_identifier = 0)
        P = (problems.slope_3d_from_mesh(coord, elem, Q) if case == "homo" else
             problems.slope_3d_from_mesh(coord, elem, Q, g[f"{case}_material"], problems.HETERO_SSR_MATERIALS))
        assert P.weight.size == 11 * elem.shape[1]
        # the element volumes (sum of |det J| w) are positive and add up to the slope's volume
        vol = P.weight.reshape(-1, 11).sum(1)
        assert np.all(vol > 0)
        assert int(Q.sum()) == g[f"{case}_sizes"][1]

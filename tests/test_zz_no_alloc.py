"""The allocation-free return mapping (sg_constitutive3d_noalloc) against sg_constitutive3d.

Two consecutive calls on the same seeded points (all five return-map branches) must each give
the same stresses, tangents and branch ids as the allocating entry point, within the FP64
tolerance of the drop-in tests (1e-12 relative per point; the two entry points run the same
kernel, so equality is expected).  A call above the stated capacity is rejected with
SG_ERR_ARG before anything runs.  This file is collected last so that the check also covers a
process in which the other GPU tests already ran.
"""
import ctypes as C

import numpy as np
import pytest

from slope_stability_octave_b200 import _lib, workloads

pytestmark = pytest.mark.gpu

MAX_POINTS = 16384  # SG_NOALLOC_MAX_POINTS in include/slopegpu.h
RTOL = 1e-12


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def run(name, d, n, want_ds=True, want_branch=True):
    S = np.zeros((n, 6))
    DS = np.zeros((n, 36)) if want_ds else None
    br = np.zeros(n, np.uint8) if want_branch else None
    args = [ptr(np.ascontiguousarray(d[k][:n])) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")]
    rc = getattr(_lib.lib(), name)(*args, n, ptr(S), ptr(DS), ptr(br))
    return rc, S, DS, br


def close(x, ref):
    nrm = np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
    return np.all(np.linalg.norm(x - ref, axis=1) <= RTOL * nrm)


def test_noalloc_matches_allocating_entry_point(cuda_device):
    d = workloads.constitutive_points(MAX_POINTS, seed=20261203)
    for n in (MAX_POINTS, 5000):
        rc, S0, DS0, b0 = run("sg_constitutive3d", d, n)
        assert rc == 0
        for _ in range(2):  # two consecutive calls reuse the same static scratch
            rc, S, DS, b = run("sg_constitutive3d_noalloc", d, n)
            assert rc == 0, _lib.lib().sg_last_error()
            assert np.array_equal(b, b0)
            assert close(S, S0) and close(DS, DS0)


@pytest.mark.parametrize("want_ds,want_branch", [(False, False), (True, False), (False, True)])
def test_noalloc_optional_outputs(cuda_device, want_ds, want_branch):
    """Stress only and/or no branch ids: the scratch is carved without the DS and branch
    regions, so S (and whichever optional output is asked for) sits at other offsets."""
    d = workloads.constitutive_points(MAX_POINTS, seed=20261204)
    n = MAX_POINTS
    rc, S0, DS0, b0 = run("sg_constitutive3d", d, n)
    assert rc == 0
    for _ in range(2):
        rc, S, DS, b = run("sg_constitutive3d_noalloc", d, n, want_ds, want_branch)
        assert rc == 0, _lib.lib().sg_last_error()
        assert close(S, S0)
        if want_ds:
            assert close(DS, DS0)
        if want_branch:
            assert np.array_equal(b, b0)


def test_noalloc_rejects_oversize(cuda_device):
    d = workloads.constitutive_points(MAX_POINTS + 1, seed=7)
    rc, _, _, _ = run("sg_constitutive3d_noalloc", d, MAX_POINTS + 1)
    assert rc == -1
    assert b"16384" in _lib.lib().sg_last_error()

"""GPU parity of the drop-in (host-buffer) entry points against the oracle.

Tolerances (FP64):
  * branch ids: bit-exact;
  * stress and tangent, per point, in the point's Frobenius norm:
        |x - x_ref| <= max(1e-12, 10 * kappa_p) * |x_ref|
    where kappa_p is the oracle's own relative change under random 1-ulp perturbations of
    the strain at that point (the reference's arithmetic sums large, nearly cancelling
    eigen-projection derivatives; at a few points per 10^5 its own result moves by up to
    ~1e-11 under 1-ulp input changes, so no implementation with different rounding can
    agree below that there).  At least 99.9 % of points must meet 1e-12 outright;
  * assembled K values: within 1e-12 relative to max |V|.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import native
from oracle.octave_ref import OctavePattern, assemble_via_oracle
from slope_stability_octave_b200 import _lib, fem, workloads

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def gpu_constitutive(dim, d, want_ds=True):
    n = d["E"].shape[0]
    ns, nds = (6, 36) if dim == 3 else (4, 9)
    S = np.zeros((n, ns))
    DS = np.zeros((n, nds)) if want_ds else None
    br = np.zeros(n, np.uint8)
    args = [ptr(np.ascontiguousarray(d[k])) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")]
    _lib.call(f"sg_constitutive{dim}d", *args, n, ptr(S), ptr(DS), ptr(br))
    return S, DS, br


def sensitivity(dim, d, draws=3):
    """Per-point relative change of the oracle's S and DS under random 1-ulp strain changes."""
    rng = np.random.default_rng(1234)
    args = [d[k] for k in ("c_bar", "sin_phi", "shear", "bulk", "lame")]
    S0, D0, _ = native.constitutive(dim, d["E"], *args)
    ks = np.zeros(len(S0))
    kd = np.zeros(len(S0))
    for _ in range(draws):
        Ep = d["E"] * (1 + rng.choice([-1.0, 1.0], size=d["E"].shape) * 2.220446049250313e-16)
        S1, D1, _ = native.constitutive(dim, Ep, *args)
        ks = np.maximum(ks, np.linalg.norm(S1 - S0, axis=1) / np.maximum(np.linalg.norm(S0, axis=1), 1e-300))
        kd = np.maximum(kd, np.linalg.norm(D1 - D0, axis=1) / np.maximum(np.linalg.norm(D0, axis=1), 1e-300))
    return ks, kd


def assert_pointwise(x, ref, kappa=None, rtol=RTOL):
    nrm = np.linalg.norm(ref, axis=1)
    err = np.linalg.norm(x - ref, axis=1)
    scale = np.maximum(nrm, np.max(nrm) * 1e-6)
    tol = rtol if kappa is None else np.maximum(rtol, 10 * kappa)
    rel = err / scale
    assert np.all(rel <= tol), f"max rel err {np.max(rel):.3e} (allowed {np.max(tol):.1e})"
    assert np.mean(rel <= rtol) >= 0.999, f"only {np.mean(rel <= rtol):.5f} of points within {rtol}"


@pytest.mark.parametrize("sorted_order", [False, True])
def test_constitutive3d_matches_oracle(cuda_device, sorted_order):
    d = workloads.constitutive_points(100_000, seed=21, sort_by_branch=sorted_order)
    S, DS, br = gpu_constitutive(3, d)
    So, DSo, bro = native.constitutive(3, d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"])
    assert np.array_equal(br, bro) and np.array_equal(br, d["target"])
    ks, kd = sensitivity(3, d)
    assert_pointwise(S, So, ks)
    assert_pointwise(DS, DSo, kd)
    # tangent symmetry is exact
    D = DS.reshape(-1, 6, 6)
    assert np.array_equal(D, D.transpose(0, 2, 1))


def test_constitutive3d_stress_only_and_odd_sizes(cuda_device):
    for n in (1, 31, 33, 1000, 70_001):
        d = workloads.constitutive_points(n, seed=n)
        S, DS, br = gpu_constitutive(3, d, want_ds=False)
        So, _, bro = native.constitutive(3, d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"], False)
        assert DS is None and np.array_equal(br, bro)
        assert_pointwise(S, So, sensitivity(3, d)[0])


def test_constitutive_empty_input(cuda_device):
    z = np.zeros(0)
    for dim in (2, 3):
        _lib.call(f"sg_constitutive{dim}d", *[ptr(z)] * 6, 0, ptr(z), ptr(z), None)


def test_constitutive2d_matches_oracle(cuda_device):
    rng = np.random.default_rng(7)
    n = 50_000
    mat = fem.elastic_fields_from_point_draws(rng.uniform(5, 15, n), rng.uniform(25, 45, n), 40000.0, 0.3)
    cb, sp = fem.davis_reduction(mat["c0"], mat["phi"], mat["psi"], 1.0)
    E = rng.normal(size=(n, 3)) * (cb / (2 * mat["shear"]))[:, None] * rng.uniform(0.1, 4, n)[:, None]
    E[: n // 6] = np.abs(E[: n // 6]) * [1, 1, 0.01]
    d = dict(E=E, c_bar=cb, sin_phi=sp, shear=mat["shear"], bulk=mat["bulk"], lame=mat["lame"])
    S, DS, br = gpu_constitutive(2, d)
    So, DSo, bro = native.constitutive(2, E, cb, sp, mat["shear"], mat["bulk"], mat["lame"])
    assert np.array_equal(br, bro)
    ks, kd = sensitivity(2, d)
    assert_pointwise(S, So, ks)
    assert_pointwise(DS, DSo, kd)


def test_constitutive3d_device_pointers(cuda_device):
    import torch
    d = workloads.constitutive_points(40_000, seed=8)
    t = {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(cuda_device) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")}
    n = d["E"].shape[0]
    S = torch.empty((n, 6), dtype=torch.float64, device=cuda_device)
    DS = torch.empty((n, 36), dtype=torch.float64, device=cuda_device)
    br = torch.empty(n, dtype=torch.uint8, device=cuda_device)
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("sg_constitutive3d_dev", *[C.c_void_p(t[k].data_ptr()) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")],
              n, C.c_void_p(S.data_ptr()), C.c_void_p(DS.data_ptr()), C.c_void_p(br.data_ptr()), C.c_void_p(st))
    torch.cuda.synchronize()
    So, DSo, bro = native.constitutive(3, d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"])
    assert np.array_equal(br.cpu().numpy(), bro)
    ks, kd = sensitivity(3, d)
    assert_pointwise(S.cpu().numpy(), So, ks)
    assert_pointwise(DS.cpu().numpy(), DSo, kd)


def test_reduction_device(cuda_device):
    import torch
    rng = np.random.default_rng(9)
    n = 10_001
    c0, phi, psi = rng.uniform(5, 15, n), np.deg2rad(rng.uniform(25, 45, n)), np.deg2rad(rng.uniform(0, 5, n))
    tc = [torch.from_numpy(a).to(cuda_device) for a in (c0, phi, psi)]
    cb = torch.empty(n, dtype=torch.float64, device=cuda_device)
    sp = torch.empty_like(cb)
    for davis in "ABC":
        _lib.call("sg_reduction_dev", *[C.c_void_p(x.data_ptr()) for x in tc], 1.37, davis.encode(), n,
                  C.c_void_p(cb.data_ptr()), C.c_void_p(sp.data_ptr()), None)
        torch.cuda.synchronize()
        rcb, rsp = fem.davis_reduction(c0, phi, psi, 1.37, davis)
        np.testing.assert_allclose(cb.cpu().numpy(), rcb, rtol=1e-13)
        np.testing.assert_allclose(sp.cpu().numpy(), rsp, rtol=1e-13)


def _assemble_case(dim, mesh):
    if dim == 3:
        xi, wf = fem.quadrature_p2_tet()
        _, a, b, c = fem.local_basis_p2_tet(xi)
        d1, d2, d3, w = fem.geometry_3d(mesh, a, b, c, wf)
        dphi, nq = (d1, d2, d3), 11
    else:
        xi, wf = fem.quadrature_p2_tri()
        _, a, b = fem.local_basis_p2_tri(xi)
        d1, d2, w = fem.geometry_2d(mesh, a, b, wf)
        dphi, nq = (d1, d2), 7
    mat = fem.materials(np.zeros(mesh.n_e, int), nq, [6, 45, 0, 40000, 0.3, 20, 20])
    pat = OctavePattern(dim, mesh.elem, mesh.n_n, dphi, w, mesh.Q, mat["shear"], mat["bulk"])
    if dim == 3:
        pts = workloads.constitutive_points(w.size, seed=31)
        _, DS, _ = native.constitutive(3, pts["E"], pts["c_bar"], pts["sin_phi"], mat["shear"], mat["bulk"], mat["lame"])
    else:
        rng = np.random.default_rng(32)
        cb, sp = fem.davis_reduction(mat["c0"], mat["phi"], mat["psi"], 1.0)
        _, DS, _ = native.constitutive(2, rng.normal(size=(w.size, 3)) * 1e-3, cb, sp, mat["shear"], mat["bulk"], mat["lame"])
    Vo, smap = assemble_via_oracle(pat, dphi, DS, nq)
    return dphi, DS, w, smap, nq, pat, Vo


@pytest.mark.parametrize("dim", [2, 3])
def test_assembly_dropin_matches_oracle(cuda_device, dim):
    mesh = fem.mesh_p2_box(4, 3, 3) if dim == 3 else fem.mesh_p2_2d(0.5, 4, 3, 4, 3, 3)
    dphi, DS, w, smap, nq, pat, Vo = _assemble_case(dim, mesh)
    V = np.zeros(pat.nnz)
    n_p = dphi[0].shape[1]
    if dim == 3:
        _lib.call("sg_assemble_ktangent3d", ptr(dphi[0]), ptr(dphi[1]), ptr(dphi[2]), ptr(DS), ptr(w), ptr(smap),
                  n_p, w.size, mesh.n_e, nq, pat.nnz, ptr(V))
    else:
        _lib.call("sg_assemble_ktangent2d", ptr(dphi[0]), ptr(dphi[1]), ptr(DS), ptr(w), ptr(smap),
                  n_p, w.size, mesh.n_e, nq, pat.nnz, ptr(V))
    assert np.max(np.abs(V - Vo)) <= RTOL * np.max(np.abs(Vo))
    # K_r values after the r-blend and symmetrisation
    Kr, Kro = pat.K_r_values(V, 0.3), pat.K_r_values(Vo, 0.3)
    assert np.max(np.abs(Kr - Kro)) <= RTOL * np.max(np.abs(Kro))


def test_assembly_rejects_out_of_range_map(cuda_device):
    mesh = fem.mesh_p2_box(2, 2, 1)
    dphi, DS, w, smap, nq, pat, Vo = _assemble_case(3, mesh)
    bad = smap.copy()
    bad[0, 0] = pat.nnz + 5
    V = np.zeros(pat.nnz)
    rc = _lib.lib().sg_assemble_ktangent3d(ptr(dphi[0]), ptr(dphi[1]), ptr(dphi[2]), ptr(DS), ptr(w), ptr(bad),
                                           10, w.size, mesh.n_e, nq, pat.nnz, ptr(V))
    assert rc == -1 and b"scatter_map" in _lib.lib().sg_last_error()

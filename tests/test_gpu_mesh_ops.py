"""GPU parity of the device mesh layer (patterns, strain, force, assembly, K_r, SpMV) against
the oracle's literal restatement of the Octave CONSTITUTIVE layer.

Pattern, transpose permutation and scatter map: bit-exact.  FP64 values: within 1e-12
relative to the largest entry (strain, force, K values, SpMV)."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import native
from oracle.octave_ref import OctavePattern
from slope_stability_octave_b200 import fem, workloads
from slope_stability_octave_b200.constitutive import CONSTITUTIVE
from slope_stability_octave_b200.device import DeviceMesh, dot, masked_diff_norm

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def build_case(kind):
    if kind == "slope3d":
        mesh = fem.mesh_p2_3d(1, 3, 2, 3, 2, 2, 3)
    elif kind == "box3d":
        mesh = fem.mesh_p2_box(3, 4, 2)
    else:
        mesh = fem.mesh_p2_2d(0.5, 4, 3, 4, 3, 3)
    if mesh.dim == 3:
        xi, wf = fem.quadrature_p2_tet()
        hat, a, b, c = fem.local_basis_p2_tet(xi)
        d1, d2, d3, w = fem.geometry_3d(mesh, a, b, c, wf)
        dphi, nq = (d1, d2, d3), 11
    else:
        xi, wf = fem.quadrature_p2_tri()
        hat, a, b = fem.local_basis_p2_tri(xi)
        d1, d2, w = fem.geometry_2d(mesh, a, b, wf)
        dphi, nq = (d1, d2), 7
    mat = fem.materials(np.zeros(mesh.n_e, int), nq, [6, 45, 0, 40000, 0.3, 20, 20])
    return mesh, dphi, w, nq, mat


def close(x, ref, rtol=RTOL):
    scale = max(np.max(np.abs(ref)), 1e-300)
    err = np.max(np.abs(np.asarray(x) - ref))
    assert err <= rtol * scale, f"rel err {err / scale:.3e}"


@pytest.mark.parametrize("kind", ["slope3d", "box3d", "slope2d"])
def test_pattern_and_maps_bitexact(cuda_device, kind):
    mesh, dphi, w, nq, mat = build_case(kind)
    dm = DeviceMesh(mesh, dphi, w, nq)
    pat = OctavePattern(mesh.dim, mesh.elem, mesh.n_n, dphi, w, mesh.Q, mat["shear"], mat["bulk"])
    I, J, tp = dm.pattern()
    assert dm.n_Q == pat.n_Q and dm.nnz_ref == pat.nnz
    assert np.array_equal(I, pat.ref_I) and np.array_equal(J, pat.ref_J)
    assert np.array_equal(tp, pat.transpose_perm)
    assert np.array_equal(dm.scatter_map(), pat.scatter_map())
    assert np.array_equal(dm.free_dofs(), pat.Q_flat)


@pytest.mark.parametrize("kind", ["slope3d", "slope2d"])
def test_strain_force_assembly_kr(cuda_device, kind):
    import torch
    mesh, dphi, w, nq, mat = build_case(kind)
    dim = mesh.dim
    dm = DeviceMesh(mesh, dphi, w, nq)
    pat = OctavePattern(dim, mesh.elem, mesh.n_n, dphi, w, mesh.Q, mat["shear"], mat["bulk"])
    cons = CONSTITUTIVE(dm, mat["c0"], mat["phi"], mat["psi"], "B", mat["shear"], mat["bulk"], mat["lame"])
    cons.init_K_r_pattern(mesh.Q)
    close(cons.V_elast_QQ(), pat.V_elast)

    rng = np.random.default_rng(3)
    U = rng.normal(size=(dim, mesh.n_n)) * 2e-3 * mesh.Q
    Ud = torch.from_numpy(np.ascontiguousarray(U.T).ravel()).to(cuda_device)
    lam = 1.1
    F = cons.build_F_and_DS_all(lam, Ud).cpu().numpy().reshape(mesh.n_n, dim).T
    # oracle: E = B U, constitutive, F = B'(w S)
    E = pat.strain(U)
    close(cons.E.cpu().numpy().reshape(-1, pat.ns), E)
    cb, spn = native.reduction(mat["c0"], mat["phi"], mat["psi"], lam, "B")
    S, DS, br = native.constitutive(dim, E, cb, spn, mat["shear"], mat["bulk"], mat["lame"])
    assert np.mean(cons.branch.cpu().numpy() == br) > 0.999
    assert len(np.unique(br)) >= 3
    Fo = pat.force(S)
    close(F, Fo, 1e-11)
    # assembly with the oracle's DS (so that branch flips at ties cannot matter)
    cons.DS.copy_(torch.from_numpy(DS.ravel()))
    r = 0.37
    I, J, V = cons.build_K_r_QQ_vals_ref(r)
    smap = pat.scatter_map()
    Vt = native.assemble(dim, dphi[0], dphi[1], dphi[2] if dim == 3 else None, DS, w, smap, nq, pat.nnz)
    close(V, pat.K_r_values(Vt, r))
    # K_t on its own (the fused K_r call does not store it on P2 tetrahedra)
    close(dm.to_ref(cons.build_K_tangent_QQ_vals()).cpu().numpy(), Vt)
    # SpMV on the free DOFs equals K(Q,Q) x; Dirichlet rows are identity
    Kq = sp.csr_matrix((V, (I - 1, J - 1)), shape=(pat.n_Q, pat.n_Q))
    x = rng.normal(size=dm.n_dof) * dm.mask.cpu().numpy()
    xd = torch.from_numpy(x).to(cuda_device)
    yd = torch.zeros_like(xd)
    dm.spmv(cons.K_r, xd, yd)
    y = yd.cpu().numpy()
    q = pat.Q_flat
    close(y[q], Kq @ x[q])
    # reductions
    assert abs(dot(xd, xd) - x @ x) <= 1e-12 * (x @ x)
    f = rng.normal(size=dm.n_dof)
    fd = torch.from_numpy(f).to(cuda_device)
    ref = np.linalg.norm((x - f)[q])
    assert abs(masked_diff_norm(xd, fd, dm.mask) - ref) <= 1e-12 * ref


def test_fused_residual_matches_three_kernel_chain(cuda_device):
    """sg_residual_dev (strain, stress-only return mapping and internal force in one kernel)
    against the chain sg_strain_dev -> sg_constitutive3d_dev -> sg_force_dev (F within 1e-12,
    branch ids equal) and against the oracle's F = B'(w S(B U)) (1e-11, as above), on a
    displacement that puts points on several plastic branches."""
    import torch
    mesh, dphi, w, nq, mat = build_case("slope3d")
    dm = DeviceMesh(mesh, dphi, w, nq)
    assert dm.fused_residual
    pat = OctavePattern(3, mesh.elem, mesh.n_n, dphi, w, mesh.Q, mat["shear"], mat["bulk"])
    cons = CONSTITUTIVE(dm, mat["c0"], mat["phi"], mat["psi"], "B", mat["shear"], mat["bulk"], mat["lame"])
    rng = np.random.default_rng(5)
    U = rng.normal(size=(3, mesh.n_n)) * 4e-3 * mesh.Q
    Ud = torch.from_numpy(np.ascontiguousarray(U.T).ravel()).to(cuda_device)
    lam = 1.4
    F_fused = cons.build_F_all(lam, Ud)
    br_fused = cons.branch.clone()
    cons.constitutive_problem_stress(Ud)
    F_chain = cons.build_F()
    assert torch.equal(br_fused, cons.branch)
    close(F_fused.cpu().numpy(), F_chain.cpu().numpy())
    E = pat.strain(U)
    cb, spn = native.reduction(mat["c0"], mat["phi"], mat["psi"], lam, "B")
    S, _, br = native.constitutive(3, E, cb, spn, mat["shear"], mat["bulk"], mat["lame"], want_ds=False)
    assert np.mean(br_fused.cpu().numpy() == br) > 0.999
    assert len(np.unique(br)) >= 3
    close(F_fused.cpu().numpy().reshape(mesh.n_n, 3).T, pat.force(S), 1e-11)


@pytest.mark.parametrize("kind", ["slope3d", "slope2d"])
def test_assembly_run_twice_and_symmetry(cuda_device, kind):
    """The tangent assembly and K_r are deterministic: two assemblies of the same DS give
    bitwise equal K_t and K_r (P2 tetrahedra: fixed summation order per block; the 2D path
    adds with FP64 atomics, whose order may vary, so there the bound is a few ulps of the
    block's magnitude), and K_r is exactly symmetric on P2 tetrahedra."""
    import torch
    mesh, dphi, w, nq, mat = build_case(kind)
    dm = DeviceMesh(mesh, dphi, w, nq)
    cons = CONSTITUTIVE(dm, mat["c0"], mat["phi"], mat["psi"], "B", mat["shear"], mat["bulk"], mat["lame"])
    cons.init_K_r_pattern(mesh.Q)
    rng = np.random.default_rng(11)
    U = rng.normal(size=(mesh.dim, mesh.n_n)) * 3e-3 * mesh.Q
    Ud = torch.from_numpy(np.ascontiguousarray(U.T).ravel()).to(cuda_device)
    cons.build_F_and_DS_all(1.2, Ud)
    Kr1 = cons.build_K_r_QQ_vals(0.3).clone()
    Kr2 = cons.build_K_r_QQ_vals(0.3).clone()
    Kt1 = cons.build_K_tangent_QQ_vals().clone()
    Kt2 = cons.build_K_tangent_QQ_vals().clone()
    if kind == "slope3d":
        assert torch.equal(Kr1, Kr2) and torch.equal(Kt1, Kt2)
        b = 3
        tr = torch.from_numpy(transpose_blocks(mesh)).to(cuda_device)
        blocks = Kr1.reshape(-1, b, b)
        assert torch.equal(blocks, blocks[tr].transpose(1, 2))
    else:
        scale = Kt1.abs().max()
        assert (Kt1 - Kt2).abs().max() <= 8 * 2.2e-16 * scale
        assert (Kr1 - Kr2).abs().max() <= 8 * 2.2e-16 * scale


def transpose_blocks(mesh):
    """Index of block (j, i) for every block (i, j) of the device pattern (the node adjacency
    with sorted rows, rebuilt on the host)."""
    from oracle.cpu_baseline import node_adjacency_csr
    A = node_adjacency_csr(mesh.elem, mesh.n_n)
    rp, col = A.indptr, A.indices
    n = rp.size - 1
    row = np.repeat(np.arange(n), np.diff(rp))
    key = row.astype(np.int64) * n + col
    tkey = col.astype(np.int64) * n + row
    order = np.argsort(key)
    return order[np.searchsorted(key[order], tkey)]


def test_assembly_staging_paths_agree(cuda_device):
    """The element blocks of P2 tetrahedra are staged by bulk copies when DS is 16-byte aligned
    and by plain loads otherwise (DS 8 bytes off a 16-byte boundary here): both give bitwise
    the same K_t, over a mesh whose last batch of eight elements is ragged, and the library's
    device status word stays clear (no bounded wait gave up)."""
    import ctypes as C

    import torch
    from slope_stability_octave_b200 import _lib
    from slope_stability_octave_b200.device import ptr
    mesh, dphi, w, nq, mat = build_case("slope3d")
    dm = DeviceMesh(mesh, dphi, w, nq)
    assert mesh.elem.shape[1] % 8 != 0
    cons = CONSTITUTIVE(dm, mat["c0"], mat["phi"], mat["psi"], "B", mat["shear"], mat["bulk"], mat["lame"])
    cons.init_K_r_pattern(mesh.Q)
    rng = np.random.default_rng(12)
    U = rng.normal(size=(mesh.dim, mesh.n_n)) * 3e-3 * mesh.Q
    Ud = torch.from_numpy(np.ascontiguousarray(U.T).ravel()).to(cuda_device)
    cons.build_F_and_DS_all(1.2, Ud)
    DS = cons.DS.contiguous()
    assert DS.data_ptr() % 16 == 0
    off = torch.empty(DS.numel() + 1, dtype=torch.float64, device=cuda_device)[1:]
    off.copy_(DS)
    assert off.data_ptr() % 16 == 8
    K1 = torch.zeros(dm.n_blocks * 9, dtype=torch.float64, device=cuda_device)
    K2 = torch.full_like(K1, float("nan"))
    dm.assemble(DS, K1)
    dm.assemble(off, K2)
    torch.cuda.synchronize()
    assert torch.equal(K1, K2)
    st = C.c_int32(-1)
    assert _lib.lib().sg_device_status(1, C.byref(st)) == 0 and st.value == 0

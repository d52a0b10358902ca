"""Kernel timings of the Newton-step hot path on one GPU (CUDA events, inputs resident).

    python -m slope_stability_octave_b200.kernel_bench [--workload box|slope|layered]
                                                       [--kernels sds,s,assembly,spmv,aorth8,aorth32,aorth64,
                                                                  vcycle64,vcycle32,amgupdate64,amgupdate32]
                                                       [--reps 20] [--order shuffled|sorted]

Workloads:
  box    the constitutive + assembly microbenchmark: structured box 80 x 40 x 40 m, 6 P2 tets
         per unit cell (768,000 tets, 1,056,321 nodes, 3,168,963 DOFs), 11-point rule
         (8,448,000 points); per-point strains seeded so that the five return-map branches
         each take 20 % (2^20 distinct seeded points repeated over the mesh), c ~ U[5,15] kPa,
         phi ~ U[25,45] deg, psi = 0, E = 40 MPa, nu = 0.3;
  slope  the 3D slope of the SSR benchmark (mesh_P2_3D(1, 15,10,15,10,10, z=40)), same draws;
  layered  the four-layer slope of the headline SSR step (mesh_P2_3D(5/3, 15,10,15,10,10,
         z=40): 1,005,075 nodes, 2,932,430 free DOFs), same draws.
The A-orthogonalisation runs against the assembled tangent of the seeded points, the AMG
kernels on the elastic stiffness of the draws' moduli.

Per kernel it prints one JSON line: mean time per launch and the algorithmic bytes per
launch (return mapping: 416 B per point with the tangent, 128 B without; assembly: 5,896 B
per element + 8 B per stored value; SpMV: 76 B per 3x3 block + row pointers + x and y), the
achieved GB/s and its fraction of the measured copy bandwidth.  Every operand is larger than
the 126 MB L2, so launches need no flush in between.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np
import torch

from . import _lib, fem, problems, workloads
from .device import DeviceMesh, cur_stream, ptr

F64 = torch.float64


def hbm_peak():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    try:
        with open(os.path.join(root, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def timed(fn, reps, warmup=3):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def build(workload):
    if workload == "box":
        mesh = workloads.box_mesh_80x40x40()
        xi, wf = fem.quadrature_p2_tet()
        _, d1, d2, d3 = fem.local_basis_p2_tet(xi)
        D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
        return mesh, (D1, D2, D3), W, wf.size
    P = problems.slope_3d_layered(5 / 3) if workload == "layered" else problems.slope_3d(1)
    return P.mesh, P.dphi, P.weight, P.n_q


def points_on_device(n, order, dev):
    """Seeded return-map inputs for n points: 2^20 distinct points (20 % per branch) tiled
    over n in a seeded random order (or grouped by branch for ``sorted``)."""
    m = min(n, 1 << 20)
    d = workloads.constitutive_points(m, seed=20261203, sort_by_branch=(order == "sorted"))
    rng = np.random.default_rng(1)
    idx = np.arange(n) % m
    idx = rng.permutation(idx) if order == "shuffled" else np.sort(idx)
    out = {}
    for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame"):
        out[k] = torch.from_numpy(np.ascontiguousarray(d[k][idx])).to(dev)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="box", choices=["box", "slope", "layered"])
    ap.add_argument("--kernels", default="sds,s,assembly,spmv")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--order", default="shuffled", choices=["shuffled", "sorted"])
    args = ap.parse_args(argv)
    kernels = args.kernels.split(",")
    dev = torch.device("cuda", torch.cuda.current_device())
    peak, peak_kind = hbm_peak()
    t0 = time.perf_counter()
    mesh, dphi, weight, n_q = build(args.workload)
    dm = DeviceMesh(mesh, dphi, weight, n_q)
    n = dm.n_int
    pts = points_on_device(n, args.order, dev)
    S = torch.empty((n, 6), dtype=F64, device=dev)
    DS = torch.empty((n, 36), dtype=F64, device=dev)
    setup_s = time.perf_counter() - t0
    L = _lib.lib()
    st = cur_stream()
    cargs = [ptr(pts[k]) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")]

    def sds():
        _lib.check(L.sg_constitutive3d_dev(*cargs, n, ptr(S), ptr(DS), None, st), "sds")

    def s_only():
        _lib.check(L.sg_constitutive3d_dev(*cargs, n, ptr(S), None, None, st), "s")

    sds()
    K = dm.new_block_values()
    x = torch.randn(dm.n_dof, dtype=F64, device=dev)
    y = torch.empty_like(x)
    nnz_vals = dm.n_blocks * 9
    base = dict(workload=args.workload, order=args.order, n_int=n, n_e=dm.n_e, n_dof=dm.n_dof,
                n_blocks=dm.n_blocks, setup_s=round(setup_s, 1), peak_gbs=peak, peak_kind=peak_kind)
    specs = {
        "sds": (sds, n * 416, "k_mc3d (S and DS)"),
        "s": (s_only, n * 128, "k_mc3d (S only)"),
        "assembly": (lambda: dm.assemble(DS, K), dm.n_e * 5896 + nnz_vals * 8,
                     "k_element_blocks_p2tet + k_gather_blocks3" if dm.tangent_fused else "k_assemble_bsr"),
        "spmv": (lambda: dm.spmv(K, x, y), dm.n_blocks * 76 + (dm.n_n + 1) * 4 + 16 * dm.n_dof,
                 "k_spmv_blk 3x3"),
    }
    dm.assemble(DS, K)

    # A-orthogonalisation of k seeded random columns against K (sg_a_orthogonalize: the
    # multi-vector SpMM A S, the Gram matrix, the recurrence, U = S T and A U = (A S) T)
    ws = {}

    def aorth(k):
        if "h" not in ws:
            h = C.c_void_p()
            _lib.call("sg_krylov_create", dm.n_dof, 100, C.byref(h))
            ws["h"] = h
            g = torch.Generator(device=dev).manual_seed(5)
            kmax = max(int(x[5:]) for x in kernels if x.startswith("aorth"))
            ws["S0"] = torch.randn((kmax, dm.n_dof), dtype=F64, device=dev, generator=g) * dm.mask
            ws["W"] = torch.empty_like(ws["S0"])
            ws["AW"] = torch.empty_like(ws["S0"])
        W = ws["W"][:k]
        W.copy_(ws["S0"][:k])
        kout = C.c_int32()
        _lib.call("sg_a_orthogonalize", ws["h"], dm.bsr, ptr(K), ptr(W), ptr(ws["AW"]), k, 1e-300, C.byref(kout),
                  st)

    # one V-cycle of the AMG preconditioner (FP64, and the mixed form's FP32 cycle) on the
    # elastic stiffness of the mesh (SPD), hierarchy and values set up once
    amgs = {}

    def vcycle(mixed):
        if mixed not in amgs:
            from .linear_solvers import AMG
            if "Kel" not in amgs:
                DSel = torch.empty_like(DS)
                dm.elastic_ds(pts["shear"], pts["bulk"], DSel)
                Kel = dm.new_block_values()
                dm.assemble(DSel, Kel)
                amgs["Kel"] = Kel
                amgs["r"] = torch.randn(dm.n_dof, dtype=F64, device=dev) * dm.mask
                amgs["z"] = torch.empty_like(amgs["r"])
            a = AMG(dm, mixed=mixed)
            a.update(amgs["Kel"])
            amgs[mixed] = a
        amgs[mixed].apply(amgs["r"], amgs["z"])

    def amg_update(mixed):
        if mixed not in amgs:
            vcycle(mixed)
        amgs[mixed].update(amgs["Kel"])

    specs["amgupdate64"] = (lambda: amg_update(False), 0, "AMG numeric value update, FP64")
    specs["amgupdate32"] = (lambda: amg_update(True), 0, "AMG numeric value update, FP32 (mixed form)")
    specs["vcycle64"] = (lambda: vcycle(False), 0, "AMG V-cycle, FP64")
    specs["vcycle32"] = (lambda: vcycle(True), 0, "AMG V-cycle, FP32 (mixed form)")
    for kk in (8, 32, 64, 128):
        # per pass of 8 columns: K once (76 B per block) + 8 columns in and out; Gram and
        # products: S, A S read, U, A U written (k columns each, 8 B per entry)
        specs[f"aorth{kk}"] = (lambda kk=kk: aorth(kk),
                               -(-kk // 8) * dm.n_blocks * 76 + 6 * kk * 8 * dm.n_dof,
                               f"sg_a_orthogonalize, k = {kk}")
    for k in kernels:
        fn, nbytes, name = specs[k]
        torch.cuda.nvtx.range_push(f"kb_{k}")      # for NVTX-filtered profiler captures
        ms = timed(fn, args.reps)
        torch.cuda.nvtx.range_pop()
        gbs = nbytes / (ms * 1e-3) / 1e9
        line = dict(base, kernel=name, ms=ms, algorithmic_bytes=nbytes, achieved_gbs=gbs, frac=gbs / peak)
        if k.startswith("vcycle") or k.startswith("amgupdate"):
            line["levels"] = amgs[k.endswith("32")].info()["levels"]
        if k == "assembly":
            line["fp64_tflops"] = dm.n_e * 71280 / (ms * 1e-3) / 1e12
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

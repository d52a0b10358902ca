#!/usr/bin/env python
"""Benchmark: seconds per SSR continuation step, 3D P2 (indirect continuation).

Workload (``config.workload``): the 3D homogeneous slope of the reference's SSR drivers,
extruded 40 m -- mesh_P2_3D(N_h = 1, 15, 10, 15, 10, 10, z = 40): 156,000 P2 tets, 220,401
nodes, 631,380 free DOFs, 1,716,000 integration points; Mohr-Coulomb (c = 6 kPa, phi = 45 deg,
psi = 0, E = 40 MPa, nu = 0.3, gamma = 20), Davis B, DFGMRES tol 1e-1 with the AMG V-cycle,
Newton tol 1e-4 (the reference scripts' settings).  Synthetic, seeded, no dataset.

A step is one accepted step of SSR_indirect_continuation (the sum of its attempts, as
stats.step_wall_time).  The init phase is untimed, W warm-up steps run untimed, then exactly
K steps are timed with CUDA events (barrier + synchronize on both sides; max over ranks).
``value`` excludes the per-step host<->device state copies; ``e2e`` includes them: every timed
step starts by copying its input state (U, U_old) from pinned host memory and ends by reading
the new state back.  The working set (K_r 441 MB, Krylov bases ~1 GB) exceeds the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form plain|mixed] [--impl reference]

Multi-GPU: replicas only (each rank runs the same continuation; no collective on the path).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s per SSR continuation step, 3D P2 (mixed+learned vs plain FP64 GPU) at equal λ"
UNIT = "s/step"
WORKLOAD = "3D homogeneous slope SSR, mesh_P2_3D(N_h=1, 15,10,15,10,10, z=40): 156,000 P2 tets, 631,380 free DOFs"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--form", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi samples (every 200 ms) during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(self.rows))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_spmv():
    """DRAM bytes per fine-level SpMV launch from the committed ncu summary (null if absent)."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as fh:
            return json.load(fh).get("spmv3_f64_dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def run_b200(args, rank, world):
    import numpy as np
    import torch

    from slope_stability_octave_b200 import _lib, problems
    from slope_stability_octave_b200.continuation import SSRIndirectStepper

    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    dev = torch.device("cuda", torch.cuda.current_device())
    t_setup = time.perf_counter()
    P = problems.slope_3d(1).to_device()
    solver = P.solver("DFGMRES_B200_MIXED" if args.form == "mixed" else "DFGMRES_B200", tol=1e-1, maxit=100)
    f = P.f_device()
    Q = P.dmesh.mask
    run = SSRIndirectStepper(problems.SSR_3D_EXTRUDED, Q, f, P.cons, solver).init()
    t_init = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        if run.step() is None:
            raise RuntimeError("continuation stopped during warm-up")
    # host-resident state for the e2e measurement
    U_h = torch.empty_like(run.U, device="cpu").pin_memory()
    Uo_h = torch.empty_like(run.U_old, device="cpu").pin_memory()
    U_h.copy_(run.U)
    Uo_h.copy_(run.U_old)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    _lib.call("sg_instr_enable", 1, 4)
    _lib.lib().sg_launch_count(1)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    steps = []
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    for k in range(args.steps):
        e0, e1, e2, e3 = ev[k]
        e0.record()
        run.U_old.copy_(Uo_h, non_blocking=True)
        run.U.copy_(U_h, non_blocking=True)
        e1.record()
        acc = run.step()
        e2.record()
        U_h.copy_(run.U, non_blocking=True)
        Uo_h.copy_(run.U_old, non_blocking=True)
        e3.record()
        if acc is None:
            raise RuntimeError("continuation stopped inside the timed region")
        steps.append(acc)
    torch.cuda.synchronize()
    launches = int(_lib.lib().sg_launch_count(1))
    ms = np.zeros(8)
    nt = np.zeros(8, np.int64)
    nl = np.zeros(8, np.int64)
    _lib.call("sg_instr_read", ms.ctypes.data_as(C.c_void_p), nt.ctypes.data_as(C.c_void_p),
              nl.ctypes.data_as(C.c_void_p), 8)
    _lib.call("sg_instr_enable", 0, 1)
    clk = clocks.stop()
    t_dev = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(args.steps)) / 1e3
    t_e2e = sum(ev[k][0].elapsed_time(ev[k][3]) for k in range(args.steps)) / 1e3
    if world > 1:
        t = torch.tensor([t_dev, t_e2e], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_dev, t_e2e = t.tolist()
    n_dof = P.dmesh.n_dof
    res = dict(t_dev=t_dev, t_e2e=t_e2e, steps=steps, launches=launches, instr=(ms, nt, nl), clocks=clk,
               n_dof=n_dof, n_blocks=P.dmesh.n_blocks, n_rows=P.dmesh.n_n, t_init=t_init,
               lam=[s["lam"] for s in steps], amg=solver.preconditioner.info())
    return res, P


def cpu_baseline_sample(P, counts, threads, log=print):
    """Reference C kernels (OpenMP) + oracle port on a z = 4 m slice of the workload (1/10 of
    its points, elements and DOFs), unit costs scaled by the size ratio, weighted by the counts
    of the timed steps."""
    import numpy as np

    from oracle.cpu_baseline import CPUSample, step_seconds
    from slope_stability_octave_b200 import problems, workloads
    from slope_stability_octave_b200.linear_solvers import near_null_space_elasticity

    S = problems.slope_3d(1, dims=(15, 10, 15, 10, 10, 4))
    # per-point strains with the branch mix of the timed steps (seeded)
    pts = workloads.constitutive_points(S.weight.size, seed=7, fractions=tuple(counts.get("branch_mix", (0.2,) * 5)))
    smp = CPUSample(S.mesh, S.dphi, S.weight, S.n_q, S.mat, pts, log=log)
    Z = near_null_space_elasticity(S.mesh.coord, S.mesh.Q)
    smp.build_amg(Z, ~S.mesh.Q.T.ravel(), log=log)
    c = smp.unit_costs()
    scale = P.dmesh.n_int / S.weight.size
    cs = {k: v * scale for k, v in c.items()}
    cs["dot"] = c["dot"] * P.dmesh.n_dof / (S.mesh.n_n * 3)
    cs["axpy"] = c["axpy"] * P.dmesh.n_dof / (S.mesh.n_n * 3)
    return step_seconds(cs, counts), dict(unit_costs_sample=c, scale=scale)


def step_counts(steps, amg_info, branch_mix=None):
    n = len(steps)
    newton = sum(s["newton_iterations_total"] for s in steps) / n
    lin = sum(s["linear_iterations"] for s in steps) / n
    return dict(newton=newton, linear=lin, damping=newton, deflation=2 * newton + 3,
                krylov_j=max(1.0, lin / max(2 * newton, 1) / 2), amg_setup_factor=3.0,
                branch_mix=branch_mix or (0.8, 0.1, 0.04, 0.04, 0.02))


def reference_arm(args, rank, world):
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    import numpy as np
    counts_path = os.path.join(ROOT, "profiles", "cfg2_step_counts.json")
    with open(counts_path) as fh:
        counts = json.load(fh)

    class _P:  # sizes of the full workload
        pass
    from slope_stability_octave_b200 import problems
    full = problems.slope_3d(1)

    class _D:
        n_int = full.weight.size
        n_dof = full.mesh.n_n * 3
    _P.dmesh = _D
    vals = []
    for i in range(args.warmup + args.steps):
        v, info = cpu_baseline_sample(_P, counts, threads, log=lambda *a: None)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.median(vals))
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=value * 1e3, higher_is_better=False, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic", impl="reference",
                config=dict(workload=WORKLOAD, form="reference CPU path", parallelism="replicas"),
                cpu_baseline=dict(value=value, unit=UNIT, cores=threads, kind="reference",
                                  sample="reference MEX kernels (OpenMP) + oracle port, z=4 m slice scaled x10, "
                                         "weighted by committed per-step counts"),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))
    return line


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        torch.distributed.init_process_group("nccl" if args.impl == "b200" else "gloo",
                                             timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    res, P = run_b200(args, rank, world)
    if rank != 0:
        return
    K = args.steps
    value_step = res["t_dev"] / K
    e2e_step = res["t_e2e"] / K
    ms, nt, nl = res["instr"]
    peak, peak_kind = peaks()
    spmv_bytes = res["n_blocks"] * (72 + 4) + (res["n_rows"] + 1) * 4 + 2 * 8 * res["n_dof"]
    spmv_ms = ms[0] / nt[0] if nt[0] else None
    achieved = spmv_bytes / (spmv_ms * 1e-3) / 1e9 if spmv_ms else None
    counts = step_counts(res["steps"], res["amg"])
    cpu = None
    if not args.no_cpu_baseline and args.gpus == 1:
        try:
            v, info = cpu_baseline_sample(P, counts, os.cpu_count() or 1, log=lambda *a: None)
            cpu = dict(value=v, unit=UNIT, cores=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                       kind="reference",
                       sample="reference MEX kernels (OpenMP, all cores) + oracle port for B*U, B'S, SpMV, MGS, "
                              "AMG V-cycle; unit costs on a z=4 m slice (1/10 of the workload) scaled by size, "
                              "weighted by the timed steps' Newton/Krylov counts")
        except Exception as exc:  # the CPU leg must not hide the GPU result
            cpu = dict(value=None, unit=UNIT, cores=None, kind="reference", sample=f"failed: {exc}")
    h2d = 2 * 8 * res["n_dof"]
    d2h = 2 * 8 * res["n_dof"]
    line = dict(
        metric=METRIC, value=value_step, unit=UNIT, n_gpus=args.gpus, steps=K, warmup=args.warmup,
        ms_per_step=value_step * 1e3, higher_is_better=False, scaling="weak", vs_baseline=None,
        dtype="f64" if args.form == "plain" else "f64 outer / f32 V-cycle", data="synthetic",
        config=dict(workload=WORKLOAD, form=args.form, parallelism=f"replicas x{args.gpus}",
                    solver="DFGMRES tol 1e-1 + AMG V-cycle", l2="working set > L2 (no flush needed)",
                    lambdas=[round(x, 8) for x in res["lam"]],
                    newton_iterations=[s["newton_iterations_total"] for s in res["steps"]],
                    linear_iterations=[s["linear_iterations"] for s in res["steps"]],
                    init_s=round(res["t_init"], 2)),
        e2e=dict(value=e2e_step, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h),
        gpu_launches=res["launches"],
        clocks=res["clocks"],
        roofline=dict(kernel="k_bsr_spmv<3,3> fine-level SpMV (FGMRES + V-cycle)", bound="hbm",
                      achieved=achieved, peak=peak, unit="GB/s", frac=(achieved / peak if achieved else None),
                      peak_kind=peak_kind, traffic=traffic_per_spmv(), algorithmic_bytes=spmv_bytes,
                      launches=int(nl[0]), timed_launches=int(nt[0]), avg_ms=spmv_ms),
        cpu_baseline=cpu,
        counts=counts,
    )
    print(json.dumps(line))


if __name__ == "__main__":
    main()

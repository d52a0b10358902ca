#!/usr/bin/env python
"""Benchmark: seconds per SSR continuation step, 3D P2 (indirect continuation).

Workloads (``--workload``, named in ``config.workload``; synthetic, seeded, no dataset):

  hetero (default, the headline)  the 3D heterogeneous slope: the reference's extruded slope
      mesh_P2_3D(N_h = 5/3, i.e. h = 0.6 m, 15, 10, 15, 10, 10, z = 40) -- 728,022 P2 tets,
      1,005,075 nodes, 2,932,430 free DOFs, 8,008,242 integration points -- with four
      horizontal material layers 5/5/10/20 m thick counted from the crest down and clipped
      at the base (c, phi, E, nu, gamma per layer: 15 kPa, 30 deg, 50 MPa, 0.3, 19 / 10, 35,
      40, 0.3, 20 / 18, 25, 60, 0.3, 21 / 6, 45, 40, 0.3, 20);
  ssr  the 3D homogeneous slope, mesh_P2_3D(N_h = 1, 15, 10, 15, 10, 10, z = 40): 156,000 P2
      tets, 220,401 nodes, 631,380 free DOFs, 1,716,000 points; c = 6 kPa, phi = 45 deg,
      psi = 0, E = 40 MPa, nu = 0.3, gamma = 20;
  ll   limit-load continuation on the slope with lognormal random-field strength at
      h = 0.45 m (see LL_WORKLOAD);
  box  the return-map microbenchmark (see BOX_WORKLOAD).

SSR workloads: Davis B, DFGMRES tol 1e-1 with the AMG V-cycle, Newton tol 1e-4 (the
reference scripts' settings).
A step is one accepted step of SSR_indirect_continuation (the sum of its attempts, as
stats.step_wall_time).  The init phase is untimed, W warm-up steps run untimed, then exactly
K steps are timed with CUDA events (barrier + synchronize on both sides; max over ranks).
The continuation state after the warm-up is kept; when the continuation reaches its end (its
factor of safety) inside the timed region, the state is restored and the timed loop goes on
with genuine accepted steps from there (``config.forms.*.replay`` lists where).
Forms, on the same workload from the same start: ``plain`` (FP64 throughout), ``mixed``
(FP32 V-cycle and AMG value updates inside the FP64 FGMRES; return mapping, Newton residual,
Arnoldi and the lambda update in FP64) and ``learned`` (mixed plus the learned node-wise
correction of the V-cycle: a per-node BF16 network trained on the GPU during the init phase
on residual vectors of the plain V-cycle, kept only if a trial solve needs fewer FGMRES
iterations and at most 95 % of the time with it).  A rejected correction leaves the learned
form equal to the mixed form; its training and trial are reported and its steps are not
timed twice.  ``value`` is the s/step of the learned form when its correction was accepted,
else of the mixed form (``config.form`` says which); per form the device time, host wall and
CPU time per step, device allocations (torch's caching allocator and the library's own
cudaMalloc count) and the lambda error against plain are in ``config.forms``.  Python's
garbage collector is paused inside the timed region.  ``value`` excludes the per-step
host<->device state copies; ``e2e`` includes them: every timed step starts by copying its
input state (U, U_old) from pinned host memory and ends by reading the new state back.  The
working set (K_r 2.0 GB on the layered slope, 441 MB on the homogeneous one; Krylov bases
several GB) exceeds the 126 MB L2, so no flush is needed between steps.  ``roofline`` is the
instrumented kernel kind with the largest share of the timed steps.

  python bench.py [--gpus N] [--steps K (20)] [--warmup W (5)] [--form all|both|plain|mixed|learned]
                  [--workload hetero|ssr|ll|box] [--impl reference] [--verbose]

Multi-GPU: replicas only (each rank runs the same continuation; no collective on the path).
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from slope_stability_octave_b200.replicas import barrier, max_over_ranks  # noqa: E402

METRIC = "s per SSR continuation step, 3D P2 (mixed+learned vs plain FP64 GPU) at equal λ"
UNIT = "s/step"
WORKLOAD = ("3D homogeneous slope SSR, mesh_P2_3D(N_h=1, 15,10,15,10,10, z=40): 156,000 P2 tets, "
            "220,401 nodes, 631,380 free DOFs, 1,716,000 integration points")
HETERO_WORKLOAD = ("3D heterogeneous slope SSR, four horizontal layers 5/5/10/20 m from the crest down, clipped at "
                   "the base (c, phi, E, nu, gamma = 15,30,50MPa,0.3,19 / 10,35,40MPa,0.3,20 / 18,25,60MPa,0.3,21 / "
                   "6,45,40MPa,0.3,20), mesh_P2_3D(N_h=5/3 i.e. h=0.6 m, 15,10,15,10,10, z=40): 728,022 P2 tets, "
                   "1,005,075 nodes, 2,932,430 free DOFs, 8,008,242 integration points")
# workload name -> (description, problem factory, CPU-sample factory (a slice of the same
# mesh, about 1/10 to 1/17 of its points), per-step counts file of the reference arm)
WORKLOADS = {
    "ssr": (WORKLOAD, lambda pb: pb.slope_3d(1), lambda pb: pb.slope_3d(1, dims=(15, 10, 15, 10, 10, 4)),
            os.path.join(ROOT, "profiles", "ssr3d_z40_step_counts.json"), "z=4 m slice (1/10)"),
    "hetero": (HETERO_WORKLOAD, lambda pb: pb.slope_3d_layered(5 / 3),
               lambda pb: pb.slope_3d_layered(5 / 3, dims=(15, 10, 15, 10, 10, 2.4)),
               os.path.join(ROOT, "profiles", "ssr3d_layered_h06_step_counts.json"), "z=2.4 m slice (4 of 67 cells)"),
}
# one-cell-deep slices of the same meshes, on which a genuine CPU continuation step is timed to
# calibrate the unit-cost model
MEASURED_SLICES = {
    "ssr": (lambda pb: pb.slope_3d(1, dims=(15, 10, 15, 10, 10, 1)), "z=1 m slice (1 of 40 cells)"),
    "hetero": (lambda pb: pb.slope_3d_layered(5 / 3, dims=(15, 10, 15, 10, 10, 0.6)), "z=0.6 m slice (1 of 67 cells)"),
}
# learned form: trained before the init phase's 4th linear solve on 12 residual vectors of
# that Newton system, 60 full-batch Adam steps
LEARNED_OPTS = dict(train_at=3, n_vectors=12, steps=60, lr=3e-3, seed=0)
N_INSTR = 12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--form", default="all", choices=["all", "both", "plain", "mixed", "learned"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="per timed step progress on stderr")
    ap.add_argument("--concurrent-solves", action="store_true",
                    help="run the two Krylov solves of each Newton step side by side (DFGMRES.solve_pair); "
                         "per-kernel timings then include the sharing of the GPU")
    ap.add_argument("--workload", default="hetero", choices=["hetero", "ssr", "ll", "box", "seepage"],
                    help="hetero: the SSR continuation step on the layered slope at h = 0.6 m (headline); ssr: the "
                         "same on the homogeneous 40 m slope at h = 1 m; ll: limit-load continuation on the "
                         "random-field slope at h = 0.45 m; box: the return-map microbenchmark")
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
        return self

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


def traffic_per_launch(kind, n_blocks):
    """DRAM bytes per launch of ``kind`` from the committed ncu summary
    (profiles/roofline_traffic.json: bytes per launch on a captured case and that case's
    block count), scaled to ``n_blocks`` blocks; null where no capture exists."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as fh:
            d = json.load(fh)
        e = d[kind]
        return e["dram_bytes_per_launch"] * n_blocks / e["blocks"]
    except (OSError, ValueError, KeyError, TypeError):
        return None


def run_form(args, form, P, rank, world):
    """One continuation of the workload in ``form``: init, W warm-up steps, K timed steps.

    The continuation stops at its factor of safety (the reference's stop tests), which on the
    benchmark slopes can come before W + K accepted steps.  The state after the warm-up is
    therefore kept (``SSRIndirectStepper.snapshot``: U, U_old, step control, histories,
    deflation basis), and when the run stops the timed loop restores it and continues with
    genuine accepted steps from there until exactly K steps are timed.  Attempts that end
    the run without an accepted step belong to no step (as in the reference's statistics)
    and are not timed; their number is reported."""
    import numpy as np
    import torch

    from slope_stability_octave_b200 import _lib, problems
    from slope_stability_octave_b200.continuation import SSRIndirectStepper
    from slope_stability_octave_b200.linear_solvers import set_linear_solver

    L = _lib.lib()
    t0 = time.perf_counter()
    solver = set_linear_solver("DFGMRES_B200" if form == "plain" else "DFGMRES_B200_MIXED", 1e-1, 100, 1e-3, 0,
                               P.dmesh, P.mesh.coord, learned=LEARNED_OPTS if form == "learned" else None, cons=P.cons)
    solver.concurrent_pair = bool(args.concurrent_solves)
    f = P.f_device()
    run = SSRIndirectStepper(problems.SSR_3D_EXTRUDED, P.dmesh.mask, f, P.cons, solver).init()
    t_init = time.perf_counter() - t0
    res = dict(t_init=t_init, lam_init=list(run.lambda_hist[:2]))
    if solver.learned is not None:
        lc = solver.learned
        res["learned"] = dict(train_s=round(lc.train_seconds, 3), trained_at_solve=lc.train_at,
                              loss_first=float(lc.loss_hist[0]), loss_last=float(lc.loss_hist[-1]),
                              params=lc.info()["nparam"], acceptance_trial=lc.gate, applied=bool(lc.enabled))
        if not lc.enabled:
            # rejected by its acceptance trial: from here on the form is the mixed form
            res["timed"] = False
            del run, solver
            gc.collect()
            return res
    for w in range(args.warmup):
        if run.step() is None:
            raise RuntimeError(f"continuation stopped during warm-up after {w} steps ({run.stop_reason})")
    snap = run.snapshot()
    snap_step = run.step_no
    # host-resident state for the end-to-end measurement
    U_h = torch.empty_like(run.U, device="cpu").pin_memory()
    Uo_h = torch.empty_like(run.U_old, device="cpu").pin_memory()
    U_h.copy_(run.U)
    Uo_h.copy_(run.U_old)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    steps, basis, host, replays, discarded, stops = [], [], [], [], 0, []
    clocks = ClockSampler(torch.cuda.current_device()).start()
    _lib.call("sg_instr_enable", 1, 4)
    # no Python garbage collection inside the timed region (a collection pass stalls the
    # launching thread while the device drains its queue)
    gc.collect()
    gc.disable()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    mem0 = torch.cuda.memory_stats()
    L.sg_launch_count(1)
    L.sg_device_alloc_count(1)
    torch.cuda.nvtx.range_push("timed_step")
    for k in range(args.steps):
        while True:
            if run.finished:
                # the continuation reached its end: replay from the post-warm-up state
                stops.append(run.stop_reason)
                run.restore(snap)
                U_h.copy_(run.U)
                Uo_h.copy_(run.U_old)
                replays.append(k)
            e0, e1, e2, e3 = ev[k]
            e0.record()
            run.U_old.copy_(Uo_h, non_blocking=True)
            run.U.copy_(U_h, non_blocking=True)
            e1.record()
            w0, c0 = time.perf_counter(), time.process_time()
            acc = run.step()
            hw = (time.perf_counter() - w0, time.process_time() - c0)
            e2.record()
            U_h.copy_(run.U, non_blocking=True)
            Uo_h.copy_(run.U_old, non_blocking=True)
            e3.record()
            if acc is not None:
                break
            discarded += 1
            if discarded > 3 * args.steps:
                raise RuntimeError(f"continuation keeps stopping without an accepted step ({run.stop_reason})")
        host.append(hw)
        steps.append(acc)
        basis.append(solver.k)
        if args.verbose:
            torch.cuda.synchronize()
            print(f"[{form}] timed step {k}: continuation step {acc['step']} lambda {acc['lam']:.8f} "
                  f"newton {acc['newton_iterations_total']} fgmres {acc['linear_iterations']} "
                  f"{ev[k][1].elapsed_time(ev[k][2]) / 1e3:.3f} s", file=sys.stderr, flush=True)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    mem1 = torch.cuda.memory_stats()
    lib_allocs = int(L.sg_device_alloc_count(1))
    gc.enable()
    barrier(world)
    launches = int(L.sg_launch_count(1))
    ms = np.zeros(N_INSTR)
    nt = np.zeros(N_INSTR, np.int64)
    nl = np.zeros(N_INSTR, np.int64)
    units = np.zeros(N_INSTR, np.int64)
    _lib.call("sg_instr_units", units.ctypes.data_as(C.c_void_p), N_INSTR)
    _lib.call("sg_instr_read", ms.ctypes.data_as(C.c_void_p), nt.ctypes.data_as(C.c_void_p),
              nl.ctypes.data_as(C.c_void_p), N_INSTR)
    _lib.call("sg_instr_enable", 0, 1)
    clk = clocks.stop()
    t_dev = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(args.steps)) / 1e3
    t_e2e = sum(ev[k][0].elapsed_time(ev[k][3]) for k in range(args.steps)) / 1e3
    t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], world, device="cuda")
    step_s = [ev[k][1].elapsed_time(ev[k][2]) / 1e3 for k in range(args.steps)]
    # device allocations inside the timed steps: torch's caching allocator and the library's own
    alloc = {k: int(mem1.get(k, 0) - mem0.get(k, 0)) for k in ("num_device_alloc", "num_device_free",
                                                              "num_alloc_retries")}
    alloc["library_device_allocs"] = lib_allocs
    # return-map branch mix of the last stress evaluation (drives the CPU-baseline sample)
    br = torch.bincount(P.cons.branch.to(torch.int64), minlength=5).double()
    res["branch_mix"] = [round(float(x), 5) for x in (br / br.sum()).cpu()]
    res.update(timed=True, t_dev=t_dev, t_e2e=t_e2e, steps=steps, step_s=step_s, alloc=alloc, host=host,
               basis=basis, launches=launches, instr=(ms, nt, nl, units), clocks=clk,
               lam=[s["lam"] for s in steps], amg=solver.preconditioner.info(),
               replay=dict(snapshot_after_step=snap_step, restored_before_timed_steps=replays,
                           stop_reasons=stops, unaccepted_attempt_runs_discarded=discarded),
               )
    if solver.learned is not None:
        res["learned"].update(fallbacks=solver.learned.fallbacks, solves=solver.learned.solves)
    del run, solver, snap
    # the caching allocator keeps its blocks for the next form, whose timed steps then run on
    # a warm allocator as a long-running solver's would (the first form warms it during its
    # own set-up); only cyclic garbage is collected here
    gc.collect()
    return res


def step_counts(res):
    """Per-step operation counts of the timed steps (drive the CPU-baseline model)."""
    steps = res["steps"]
    n = len(steps)
    newton = sum(s["newton_iterations_total"] for s in steps) / n
    lin = sum(s["linear_iterations"] for s in steps) / n
    return dict(newton=newton, linear=lin, damping=newton, deflation=sum(res["basis"]) / n,
                krylov_j=max(1.0, lin / max(2 * newton, 1) / 2),
                branch_mix=tuple(res.get("branch_mix", (0.8, 0.1, 0.04, 0.04, 0.02))))


def cpu_sample(workload="ssr", log=lambda *a: None, branch_mix=(0.8, 0.1, 0.04, 0.04, 0.02)):
    """The CPU path's unit costs are timed on a slice of the workload (the same mesh spacing
    and material, a few cells deep in z) and scaled by the size ratio; the return mapping runs
    on seeded points with the timed GPU steps' branch mix."""
    import numpy as np

    from oracle.cpu_baseline import CPUSample
    from slope_stability_octave_b200 import problems, workloads
    from slope_stability_octave_b200.linear_solvers import near_null_space_elasticity

    S = WORKLOADS[workload][2](problems)
    mix = np.asarray(branch_mix, float)
    pts = workloads.constitutive_points(S.weight.size, seed=7, fractions=tuple(mix / mix.sum()))
    smp = CPUSample(S.mesh, S.dphi, S.weight, S.n_q, S.mat, pts, log=log)
    Z = near_null_space_elasticity(S.mesh.coord, S.mesh.Q)
    smp.build_amg(Z, ~S.mesh.Q.T.ravel(), log=log)
    return S, smp


def cpu_step_seconds(S, smp, counts, n_int_full, n_dof_full):
    from oracle.cpu_baseline import step_seconds
    c = smp.unit_costs()
    scale = n_int_full / S.weight.size
    cs = {k: v * scale for k, v in c.items()}
    cs["dot"] = c["dot"] * n_dof_full / (S.mesh.n_n * 3)
    cs["axpy"] = c["axpy"] * n_dof_full / (S.mesh.n_n * 3)
    return step_seconds(cs, counts), c


def cpu_calibration(workload, branch_mix=(0.8, 0.1, 0.04, 0.04, 0.02), log=lambda *a: None):
    """One genuine CPU continuation step (after an untimed init phase) on the one-cell slice,
    and the unit-cost model of the same slice with that step's own counts: returns
    (measured / model, details).  The CPU path: the oracle's Newton and continuation drivers,
    the reference's return mapping restated in C and the assembly, DFGMRES with the oracle's
    AMG V-cycle on the host (oracle.cpu_baseline.HostAMGDFGMRES)."""
    import numpy as np

    from oracle.cpu_baseline import CPUSample, measured_steps, step_seconds
    from slope_stability_octave_b200 import problems, workloads
    from slope_stability_octave_b200.linear_solvers import near_null_space_elasticity
    S1 = MEASURED_SLICES[workload][0](problems)
    st = measured_steps(S1, problems.SSR_3D_EXTRUDED, n_steps=1, log=log)
    wall = st["step_wall_time"][0]
    newton = st["step_newton_iterations"][0]
    lin = st["step_linear_iterations"][0]
    mix = np.asarray(branch_mix, float)
    pts = workloads.constitutive_points(S1.weight.size, seed=7, fractions=tuple(mix / mix.sum()))
    smp = CPUSample(S1.mesh, S1.dphi, S1.weight, S1.n_q, S1.mat, pts, log=log)
    smp.build_amg(near_null_space_elasticity(S1.mesh.coord, S1.mesh.Q), ~S1.mesh.Q.T.ravel(), log=log)
    counts = dict(newton=newton, linear=lin, damping=newton, deflation=max(st["deflation"], 1),
                  krylov_j=max(1.0, lin / max(2 * newton, 1) / 2))
    model = step_seconds(smp.unit_costs(), counts)
    return wall / model, dict(measured_slice_step_s=round(wall, 3), model_slice_step_s=round(model, 3),
                              measured_over_model=round(wall / model, 3), slice=MEASURED_SLICES[workload][1],
                              slice_free_dofs=int(S1.mesh.Q.sum()), slice_points=int(S1.weight.size),
                              slice_counts=dict(newton=newton, linear=lin, deflation=st["deflation"]))


def cpu_sample_text(workload="ssr"):
    return ("one continuation step of the CPU path, modelled and calibrated: unit costs of every Newton-iteration "
            f"operation timed on a {WORKLOADS[workload][4]} of the workload and scaled by size, weighted by the "
            "timed GPU steps' Newton/Krylov/deflation counts, times the measured/model ratio of one genuine CPU "
            f"continuation step timed on a {MEASURED_SLICES[workload][1]} (calibration); return mapping and tangent "
            "assembly are the reference's own C (MEX sources compiled with -O2 -fopenmp, all host threads), B*U, B'S, "
            "SpMV, Gram-Schmidt, deflation and the AMG set-up/V-cycle are the NumPy/SciPy port (single-threaded "
            "except SciPy's compiled kernels; the reference's Octave/sparsersb/HYPRE layer is not installable)")


def reference_arm(args, rank, world):
    """The reference's CPU path on the host cores: every step re-times the unit costs of the
    operations of a Newton iteration on the slice and evaluates the calibrated model of one
    full-size continuation step (counts of the GPU plain form's timed steps, committed in
    profiles/); the calibration (one genuine CPU continuation step on a one-cell slice
    against the model of that slice) runs once before the warm-up."""
    if rank != 0:
        return None
    import numpy as np
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    desc, _, _, counts_file, _ = WORKLOADS[args.workload]
    with open(counts_file) as fh:
        counts = json.load(fh)
    t0 = time.perf_counter()
    mix = counts.get("branch_mix", (0.8, 0.1, 0.04, 0.04, 0.02))
    ratio, calib = cpu_calibration(args.workload, branch_mix=mix)
    S, smp = cpu_sample(args.workload, branch_mix=mix)
    t_setup = time.perf_counter() - t0
    vals, models = [], []
    t1 = time.perf_counter()
    for i in range(args.warmup + args.steps):
        v, _ = cpu_step_seconds(S, smp, counts, counts["n_int"], counts["n_dof"])
        if i >= args.warmup:
            models.append(v)
            vals.append(v * ratio)
    value = float(np.mean(vals))
    calib.update(model_full_step_s=round(float(np.mean(models)), 2), setup_s=round(t_setup, 1),
                 unit_cost_loop_s=round(time.perf_counter() - t1, 1))
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=value * 1e3, higher_is_better=False, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic", impl="reference",
                config=dict(workload=desc, form="reference CPU path (plain FP64)", parallelism="replicas",
                            counts=counts, calibration=calib,
                            timing="a step is one evaluation of the calibrated step model (unit costs re-timed "
                                   "each step); the full-size CPU step itself (minutes) is not run"),
                cpu_baseline=dict(value=value, unit=UNIT, cores=int(os.environ["OMP_NUM_THREADS"]), kind="port",
                                  sample=cpu_sample_text(args.workload)),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))
    return line


LL_METRIC = "s per LL continuation step, 3D P2 random-field slope (mixed vs plain FP64 GPU) at equal step"
LL_WORKLOAD = ("3D limit-load (LL) indirect continuation on the extruded slope with lognormal random-field strength "
               "(c mean 10 kPa CoV 0.3, phi mean 35 deg CoV 0.1, independent, exponential correlation 5 m, circulant "
               "embedding on a 0.5 m grid, seed 20261203; E = 40 MPa, nu = 0.3, gamma = 20), mesh_P2_3D(N_h=20/9 "
               "i.e. h=0.45 m, 15,10,15,10,10, z=40)")


def run_ll_form(args, form, P):
    """Elastic start, then W + K accepted steps of LL_indirect_continuation; the last K are
    timed (sum of attempt wall times with the device synchronised around each attempt)."""
    import torch

    from slope_stability_octave_b200 import continuation, problems
    from slope_stability_octave_b200.linear_solvers import set_linear_solver

    p = problems.LL_3D_EXTRUDED
    t0 = time.perf_counter()
    solver = set_linear_solver("DFGMRES_B200" if form == "plain" else "DFGMRES_B200_MIXED", 1e-1, 100, 1e-3, 0,
                               P.dmesh, P.mesh.coord, learned=LEARNED_OPTS if form == "learned" else None, cons=P.cons)
    solver.concurrent_pair = bool(args.concurrent_solves)
    f = P.f_device()
    Q = P.dmesh.mask
    U0, d_omega = continuation.LL_elastic_start(Q, f, P.cons, solver)
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t0
    _, th, oh, _, st = continuation.LL_indirect_continuation(
        d_omega, p["d_t_min"], p["step_max"], p["omega_max"], p["it_newt_max"], p["it_damp_max"], p["tol"],
        p["r_min"], None, U0, Q, f, P.cons, solver.copy(), max_steps=args.warmup + args.steps)
    n = len(st["step_wall_time"])
    if n < args.warmup + args.steps:
        raise RuntimeError(f"LL continuation stopped after {n} steps ({st['stop_reason']})")
    timed = st["step_wall_time"][args.warmup:]
    res = dict(t=list(th[1:]), omega=list(oh[1:]), newton=st["step_newton_iterations"],
               linear=st["step_linear_iterations"], attempts=st["attempts"], wall=st["step_wall_time"],
               s_per_step=sum(timed) / len(timed), init_s=round(t_init, 2))
    del solver
    gc.collect()
    return res


def run_ll(args, rank, world):
    import torch

    from slope_stability_octave_b200 import problems
    t0 = time.perf_counter()
    P = problems.slope_3d_random_field(20 / 9).to_device()
    t_setup = time.perf_counter() - t0
    forms = {"all": ["plain", "mixed", "learned"], "both": ["plain", "mixed"]}.get(args.form, [args.form])
    clocks = ClockSampler(torch.cuda.current_device()).start()
    out = {form: run_ll_form(args, form, P) for form in forms}
    clk = clocks.stop()
    if rank != 0:
        return
    head_form = "mixed" if "mixed" in out else forms[0]
    m = P.mesh
    cfg = dict(workload=LL_WORKLOAD, mesh=dict(tets=m.n_e, nodes=m.n_n, free_dofs=int(m.Q.sum()),
                                               points=int(P.weight.size)),
               random_field=m.info.get("random_field"), setup_s=round(t_setup, 1), form=head_form,
               timing="sum of attempt wall times per accepted step, device synchronised around each attempt",
               forms=out)
    for other in ("mixed", "learned"):
        if "plain" in out and other in out:
            tp, tm = out["plain"]["t"], out[other]["t"]
            cfg[f"t_rel_err_{other}_vs_plain"] = max(abs(a - b) / abs(a) for a, b in zip(tp, tm))
            cfg[f"speedup_{other}_vs_plain"] = out["plain"]["s_per_step"] / out[other]["s_per_step"]
    v = out[head_form]["s_per_step"]
    line = dict(metric=LL_METRIC, value=v, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=v * 1e3, higher_is_better=False, scaling="weak", vs_baseline=None,
                dtype="f64 (f32 V-cycle)" if head_form != "plain" else "f64", data="synthetic (seeded random field)",
                config=cfg, clocks=clk)
    print(json.dumps(line))


BOX_METRIC = ("ms per constitutive + assembly pass (S, DS and the B'DB tangent K_t), structured box 80x40x40 m, "
              "8,448,000 points, 768,000 P2 tets")
BOX_WORKLOAD = ("box 80x40x40 m, 6 P2 tets per unit cell (768,000 tets, 1,056,321 nodes), 11-point rule: 8,448,000 "
                "points; seeded strains with the five return-map branches at 20 % each in random order; c ~ U[5,15] "
                "kPa, phi ~ U[25,45] deg, psi = 0, E = 40 MPa, nu = 0.3; K_t assembled into the node-block pattern "
                "of the mesh from the pass's DS")
BOX_SAMPLE = 1 << 20
BOX_ASM_SAMPLE = (16, 16, 16)   # cells of the small box whose assembly the CPU sample times


def box_cpu_ms(n_full, threads, reps=3):
    """The reference's own return-map MEX (oracle/_ref, OpenMP on all host threads) on the
    first 2^20 points of the same seeded set, scaled to the full point count."""
    from oracle import native
    from slope_stability_octave_b200 import workloads
    d = workloads.constitutive_points(BOX_SAMPLE, seed=20261203)
    args = (d["E"], d["c_bar"], d["sin_phi"], d["shear"], d["bulk"], d["lame"])
    native.ref_constitutive(3, *args, want_ds=True)
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        native.ref_constitutive(3, *args, want_ds=True)
        best = min(best, time.perf_counter() - t0)
    return best * 1e3 * n_full / BOX_SAMPLE


_ASM_SAMPLE = {}


def box_cpu_assembly_ms(n_e_full, reps=3):
    """The reference's own tangent assembly MEX (assemble_K_tangent_vals.c compiled from its
    sources, OpenMP on all host threads, int64 scatter map in find() order) on the 16x16x16-cell
    box (24,576 tets) with seeded tangents, scaled per element to the full box."""
    import numpy as np

    from oracle import native
    from oracle.cpu_baseline import CPUSample
    from slope_stability_octave_b200 import fem, workloads
    if "smp" not in _ASM_SAMPLE:
        mesh = fem.mesh_p2_box(*BOX_ASM_SAMPLE, 1.0)
        xi, wf = fem.quadrature_p2_tet()
        _, d1, d2, d3 = fem.local_basis_p2_tet(xi)
        D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
        mat = fem.materials(np.zeros(mesh.n_e, int), wf.size, [[10.0, 35.0, 0.0, 40000.0, 0.3, 20.0, 20.0]])
        pts = workloads.constitutive_points(W.size, seed=5)
        smp = CPUSample(mesh, (D1, D2, D3), W, wf.size, mat, pts, log=lambda *a: None)
        _, DS = native.ref_constitutive(3, pts["E"], pts["c_bar"], pts["sin_phi"], pts["shear"], pts["bulk"],
                                        pts["lame"], want_ds=True)
        _ASM_SAMPLE.update(smp=smp, DS=DS, n_e=mesh.n_e, dphi=(D1, D2, D3), W=W, nq=wf.size)
    a = _ASM_SAMPLE
    smp = a["smp"]
    run = lambda: native.ref_assemble(3, a["dphi"][0], a["dphi"][1], a["dphi"][2], a["DS"], a["W"], smp.smap,
                                      a["nq"], smp.nnz)
    run()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        run()
        best = min(best, time.perf_counter() - t0)
    return best * 1e3 * n_e_full / a["n_e"]


def run_box(args, rank):
    """Constitutive + assembly microbenchmark: per pass, S and DS for every point of the box and
    the tangent K_t assembled from that DS into the mesh's block pattern, inputs resident
    (value); the drop-in host-buffer return map with its copies (e2e)."""
    import numpy as np
    import torch

    from slope_stability_octave_b200 import _lib, fem
    from slope_stability_octave_b200.device import DeviceMesh, cur_stream, ptr
    from slope_stability_octave_b200.kernel_bench import points_on_device
    from slope_stability_octave_b200.workloads import box_mesh_80x40x40

    dev = torch.device("cuda", torch.cuda.current_device())
    mesh = box_mesh_80x40x40()
    xi, wf = fem.quadrature_p2_tet()
    _, d1, d2, d3 = fem.local_basis_p2_tet(xi)
    D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
    dm = DeviceMesh(mesh, (D1, D2, D3), W, wf.size)
    n = dm.n_int
    pts = points_on_device(n, "shuffled", dev)
    S = torch.empty((n, 6), dtype=torch.float64, device=dev)
    DS = torch.empty((n, 36), dtype=torch.float64, device=dev)
    K = dm.new_block_values()
    L = _lib.lib()
    st = cur_stream()
    cargs = [ptr(pts[k]) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")]

    def sds():
        _lib.check(L.sg_constitutive3d_dev(*cargs, n, ptr(S), ptr(DS), None, st), "sg_constitutive3d_dev")

    def assemble():
        _lib.check(L.sg_assemble_bsr_dev(dm.handle, ptr(DS), ptr(K), st), "sg_assemble_bsr_dev")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record()
    for _ in range(args.warmup):
        sds()
        assemble()
    w1.record()
    torch.cuda.synchronize()
    # a pass takes ~10 ms: the K timed passes are repeated in rounds until the timed region
    # spans >= 3 s, so the clock sampler (every 200 ms) sees it; every pass is timed
    per_pass = w0.elapsed_time(w1) / max(args.warmup, 1)
    rounds = max(1, int(np.ceil(3000.0 / max(per_pass * args.steps, 1e-3))))
    rounds = int(max_over_ranks([float(rounds)], world, device="cuda")[0])
    barrier(world)
    clocks = ClockSampler(torch.cuda.current_device()).start()
    L.sg_launch_count(1)
    n_pass = rounds * args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(n_pass)]
    for k in range(n_pass):
        ev[k][0].record()
        sds()
        ev[k][1].record()
        assemble()
        ev[k][2].record()
    torch.cuda.synchronize()
    launches = int(L.sg_launch_count(1))
    clk = clocks.stop()
    barrier(world)
    t_sds = sum(e[0].elapsed_time(e[1]) for e in ev) / n_pass
    t_asm = sum(e[1].elapsed_time(e[2]) for e in ev) / n_pass
    t_sds, t_asm = max_over_ranks([t_sds, t_asm], world, device="cuda")
    ms = t_sds + t_asm
    if rank != 0:
        return
    # e2e: the drop-in host-buffer return map (the MEX arguments), copies included, plus the
    # device assembly of its DS
    host = {k: pts[k].cpu().numpy() for k in pts}
    Sh = np.empty((n, 6))
    DSh = np.empty((n, 36))
    hargs = [host[k].ctypes.data_as(C.c_void_p) for k in ("E", "c_bar", "sin_phi", "shear", "bulk", "lame")]
    _lib.call("sg_constitutive3d", *hargs, n, Sh.ctypes.data_as(C.c_void_p), DSh.ctypes.data_as(C.c_void_p), None)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _lib.call("sg_constitutive3d", *hargs, n, Sh.ctypes.data_as(C.c_void_p), DSh.ctypes.data_as(C.c_void_p),
                  None)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps + t_asm
    peak, peak_kind = peaks()
    b_sds = n * 416
    b_asm = dm.n_e * 5896 + dm.n_blocks * 72
    ach_sds = b_sds / (t_sds * 1e-3) / 1e9
    ach_asm = b_asm / (t_asm * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        os.environ.setdefault("OMP_NUM_THREADS", str(threads))
        c_sds = box_cpu_ms(n, threads)
        c_asm = box_cpu_assembly_ms(dm.n_e)
        cpu = dict(value=c_sds + c_asm, unit="ms/pass", cores=int(os.environ["OMP_NUM_THREADS"]), kind="reference",
                   return_map_ms=c_sds, assembly_ms=c_asm,
                   sample="reference constitutive_problem_3D_SDS_mex on the first 2^20 points of the seeded set "
                          "(scaled to 8,448,000 points) + reference assemble_K_tangent_vals on a 16x16x16-cell box "
                          "(24,576 tets, scaled per element to 768,000), both compiled from their sources with "
                          "-O2 -fopenmp, best of 3")
    rows = {"return_map": dict(kernel="k_mc3d<S and DS>", ms=t_sds, algorithmic_bytes=b_sds, achieved=ach_sds,
                               frac=ach_sds / peak),
            "assembly": dict(kernel="k_element_blocks_p2tet + k_gather_blocks3 (deterministic B'DB)", ms=t_asm,
                             algorithmic_bytes=b_asm, achieved=ach_asm, frac=ach_asm / peak,
                             fp64_tflops=dm.n_e * 71280 / (t_asm * 1e-3) / 1e12)}
    top = max(rows, key=lambda k: rows[k]["ms"])
    r = rows[top]
    line = dict(metric=BOX_METRIC, value=ms, unit="ms/pass", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=ms, higher_is_better=False, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic (seeded points)",
                config=dict(workload=BOX_WORKLOAD, l2="3.5 GB per return-map pass, 4.5 GB of assembly inputs > L2 "
                                                      "(no flush needed)", parts=rows, tets=dm.n_e,
                            blocks=dm.n_blocks, timed_passes=n_pass,
                            timing=f"{rounds} rounds of the {args.steps} timed passes (the timed region spans >= 3 s "
                                   "for the clock record); CUDA events around each part of every pass"),
                e2e=dict(value=e2e_ms, unit="ms/pass", h2d_bytes_per_step=n * 80, d2h_bytes_per_step=n * 336),
                gpu_launches=launches, clocks=clk,
                roofline=dict(kernel=r["kernel"], bound="hbm", achieved=r["achieved"], peak=peak, unit="GB/s",
                              frac=r["frac"], peak_kind=peak_kind, traffic=None,
                              algorithmic_bytes_per_launch=r["algorithmic_bytes"]),
                cpu_baseline=cpu)
    print(json.dumps(line))


def box_reference_arm(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    vals = []
    for i in range(args.warmup + args.steps):
        v = box_cpu_ms(8448000, threads, reps=1) + box_cpu_assembly_ms(768000, reps=1)
        if i >= args.warmup:
            vals.append(v)
    value = sum(vals) / len(vals)
    line = dict(metric=BOX_METRIC, value=value, unit="ms/pass", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=value, higher_is_better=False, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic (seeded points)", impl="reference",
                config=dict(workload=BOX_WORKLOAD),
                cpu_baseline=dict(value=value, unit="ms/pass", cores=int(os.environ["OMP_NUM_THREADS"]),
                                  kind="reference",
                                  sample="constitutive_problem_3D_SDS_mex on 2^20 points, scaled to 8,448,000, plus "
                                         "assemble_K_tangent_vals on a 16x16x16-cell box, scaled to 768,000 tets"),
                e2e=dict(value=value, unit="ms/pass", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))


KINDS = ["spmv3_f64", "spmv3_f32", "constitutive_S_DS", "constitutive_S", "assembly", "amg_update", "amg_vcycle",
         "spmv3_f16", "spmv3_f64_aorth", "residual", "spmm3_f64_aorth", "a_orthogonalize"]
KIND_NAMES = {
    "spmv3_f64": "k_spmv_blk 3x3 FP64, fine level (Arnoldi, projection, residuals)",
    "spmv3_f32": "k_spmv_blk 3x3 FP32, fine level of the FP32 V-cycle",
    "constitutive_S_DS": "k_mc3d return mapping + tangent",
    "constitutive_S": "k_mc3d return mapping (stress only)",
    "assembly": "tangent assembly (B'DB into the block pattern)",
    "amg_update": "AMG numeric value update (sequence of kernels per Newton iteration)",
    "amg_vcycle": "AMG V-cycle (sequence of kernels per application)",
    "spmv3_f16": "k_spmv_h3 FP16 level-0 copy",
    "spmv3_f64_aorth": "k_spmv_blk 3x3 FP64 inside the A-orthogonalisation",
    "residual": "k_residual3d fused stress-only residual",
    "spmm3_f64_aorth": "k_spmm3 FP64 multi-vector SpMM of the A-orthogonalisation",
    "a_orthogonalize": "whole A-orthogonalisation of the deflation basis (SpMM + blocked Gram-Schmidt)",
}


def kind_bytes(P, amg, units=None, launches=None):
    """Algorithmic bytes per launch of every instrumented kind (each operand read once, each
    result written once).  SpMV: values + block columns + row pointers + x read + y written;
    return map 416 B (S and DS) or 128 B (S) per point; assembly 5,896 B per element + the K
    values written; fused residual 280 B per point + U gathered and F written once; AMG
    update: the fine matrix read (and its FP32 copy written in the mixed form), every level's
    P and R written, every coarse matrix written; V-cycle: per level six smoother/residual
    SpMVs and the two transfers, the coarsest dense solve."""
    dm = P.dmesh
    nb, nr, nd, ni, ne = dm.n_blocks, dm.n_n, dm.n_dof, dm.n_int, P.mesh.n_e
    s = 4 if amg.get("mixed") else 8
    lv = amg["levels"]
    spmv64 = nb * (72 + 4) + (nr + 1) * 4 + 2 * 8 * nd
    upd = nb * (72 + 4) + (nb * 36 if s == 4 else 0)
    cyc = 0
    for i, l in enumerate(lv):
        b = l["block"]
        if i + 1 < len(lv):
            bc = lv[i + 1]["block"]
            upd += 2 * l["p_blocks"] * b * bc * s + lv[i + 1]["blocks"] * bc * bc * s
            a_bytes = l["blocks"] * (b * b * s + 4) + (l["rows"] + 1) * 4 + 3 * l["rows"] * b * s
            cyc += 6 * a_bytes + 2 * (l["p_blocks"] * (b * bc * s + 4) + (l["rows"] + 1) * 4)
        else:
            cyc += amg["coarse_dense"] ** 2 * s
    # SpMM: the matrix once per launch, every vector of the launch read and written once
    kc = (units[10] / launches[10]) if units is not None and launches is not None and launches[10] else 1.0
    spmm = nb * (72 + 4) + (nr + 1) * 4 + 2 * 8 * nd * kc
    return {"spmv3_f64": spmv64, "spmv3_f64_aorth": spmv64, "spmm3_f64_aorth": spmm,
            "spmv3_f32": nb * (36 + 4) + (nr + 1) * 4 + 3 * 4 * nd,
            "spmv3_f16": nb * (24 + 4) + (nr + 1) * 4 + 3 * 4 * nd,
            "constitutive_S_DS": ni * 416, "constitutive_S": ni * 128,
            "assembly": ne * 5896 + nb * 72, "residual": ni * 280 + ne * 30 * 8 + nd * 8,
            "amg_update": upd, "amg_vcycle": cyc, "a_orthogonalize": None}


def roofline_report(head, kbytes, K, peak, peak_kind, n_blocks):
    """Roofline of the kind with the largest share of the timed steps (live CUDA-event samples
    of every 4th launch), with every other instrumented kind beside it."""
    ms, nt, nl = head["instr"][:3]
    total = head["t_dev"] * 1e3
    rows = {}
    for i, name in enumerate(KINDS):
        if not nl[i] or not nt[i]:
            continue
        avg = ms[i] / nt[i]
        row = dict(kernel=KIND_NAMES[name], launches=int(nl[i]), timed_launches=int(nt[i]), avg_ms=avg,
                   share_of_timed_steps=avg * nl[i] / total)
        if kbytes.get(name) is not None:
            ach = kbytes[name] / (avg * 1e-3) / 1e9
            row.update(algorithmic_bytes_per_launch=int(kbytes[name]), achieved=ach, frac=ach / peak)
        else:
            units = head["instr"][3][i]
            row["mean_units_per_launch"] = float(units) / nl[i] if nl[i] else None
        rows[name] = row
    top = max((k for k in rows if "achieved" in rows[k]), key=lambda k: rows[k]["share_of_timed_steps"])
    r = rows[top]
    return dict(kernel=r["kernel"], kind=top, bound="hbm", achieved=r["achieved"], peak=peak, unit="GB/s",
                frac=r["frac"], peak_kind=peak_kind, traffic=traffic_per_launch(top, n_blocks),
                algorithmic_bytes_per_launch=r["algorithmic_bytes_per_launch"], launches=r["launches"],
                timed_launches=r["timed_launches"], avg_ms=r["avg_ms"], share=r["share_of_timed_steps"],
                other_kernels={k: v for k, v in rows.items() if k != top})



SEEPAGE_METRIC = "s per seepage solve (initial linear solve + damped Newton to 1e-10), 3D P2 slope with phreatic line"
SEEPAGE_WORKLOAD = ("unconfined seepage of slope_stability_3D_homo_seepage_SSR.m (k = 1, phreatic line y21 = 2 m at the "
                    "face, y22 = 6 m higher at x = 0, penalty eps = grho h_min / 2) on mesh_P2_3D(N_h=1, 15,10,15,10,10, "
                    "z=40): 156,000 P2 tets, 220,401 pressure nodes; DFGMRES tol 1e-6 (200 iterations) with the scalar "
                    "AMG V-cycle, as the script's seepage solver")
SEEPAGE_SAMPLE_DIMS = (15, 10, 15, 10, 10, 1)


def seepage_problem_inputs(dims):
    import numpy as np

    from slope_stability_octave_b200 import fem, problems
    mesh = fem.mesh_p2_3d(1, *dims)
    xi, wf = fem.quadrature_p2_tet()
    hat, d1, d2, d3 = fem.local_basis_p2_tet(xi)
    D1, D2, D3, W = fem.geometry_3d(mesh, d1, d2, d3, wf)
    Q_w, pw_D = problems.homo_slope_seepage_bc(mesh.coord, *dims[:5])
    return mesh, hat, (D1, D2, D3), W, wf.size, Q_w, pw_D, np.ones(mesh.n_e * wf.size)


def seepage_cpu_seconds(reps=1):
    """The oracle's seepage solve (sparse direct solves) on a z = 1 m slice of the workload,
    scaled by the node count to the full mesh; one host thread for the sparse LU."""
    from oracle import seepage_ref as sr
    mesh, hat, dphi, W, n_q, Q_w, pw_D, conduct = seepage_problem_inputs(SEEPAGE_SAMPLE_DIMS)
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        sr.seepage_problem(mesh.coord, mesh.elem, Q_w, pw_D, sr.GRHO, conduct, hat, dphi, W)
        best = min(best, time.perf_counter() - t0)
    return best, mesh.n_n


def run_seepage(args, rank):
    """K timed seepage solves from scratch (W warm-up solves before): each solve uploads its
    inputs (Dirichlet pressure, conductivity per point, penalty per element), runs the initial
    linear solve and the damped Newton on the device and, for e2e, copies the pressure back.
    value: CUDA-event time of the solves; e2e: host wall time with the copies."""
    import numpy as np
    import torch

    from slope_stability_octave_b200 import _lib, seepage
    from slope_stability_octave_b200.device import DeviceMesh
    mesh, hat, dphi, W, n_q, Q_w, pw_D, conduct = seepage_problem_inputs((15, 10, 15, 10, 10, 40))
    dm = DeviceMesh(mesh, dphi, W, n_q)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    out_h = torch.empty(mesh.n_n, dtype=torch.float64).pin_memory()
    stats = []

    def solve(e2e):
        solver = seepage.seepage_solver(dm, Q_w)
        pw, grad_p, sat, st = seepage.seepage_problem(dm, hat, Q_w, pw_D, conduct, solver=solver)
        if e2e:
            out_h.copy_(pw)
        stats.append(st)
        return pw

    for _ in range(args.warmup):
        solve(False)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(torch.cuda.current_device()).start()
    L = _lib.lib()
    L.sg_launch_count(1)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        solve(False)
    b.record()
    torch.cuda.synchronize()
    launches = int(L.sg_launch_count(1))
    t_dev = a.elapsed_time(b) / 1e3 / args.steps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        solve(True)
    torch.cuda.synchronize()
    t_e2e = (time.perf_counter() - t0) / args.steps
    clk = clocks.stop()
    t_dev = max_over_ranks([t_dev], world, device="cuda")[0]
    if rank != 0:
        return
    st = stats[-1]
    cpu = None
    if not args.no_cpu_baseline:
        c_s, n_sample = seepage_cpu_seconds()
        cpu = dict(value=c_s * mesh.n_n / n_sample, unit="s/solve", cores=1, kind="port",
                   sample=f"the oracle's seepage solve (SciPy sparse LU) on the z = 1 m slice ({n_sample} nodes, "
                          f"{c_s:.2f} s), scaled by the node count to {mesh.n_n} nodes")
    line = dict(metric=SEEPAGE_METRIC, value=t_dev, unit="s/solve", n_gpus=args.gpus, steps=args.steps,
                warmup=args.warmup, ms_per_step=t_dev * 1e3, higher_is_better=False, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic (generated mesh)",
                config=dict(workload=SEEPAGE_WORKLOAD, nodes=mesh.n_n, tets=mesh.n_e, free_nodes=int(Q_w.sum()),
                            newton_iterations=st["iterations"], linear_iterations=st["linear_iterations"],
                            initial_linear_iterations=st["initial_linear_iterations"], status=st["status"],
                            l2="working set > L2 on the Krylov bases; no flush"),
                e2e=dict(value=t_e2e, unit="s/solve",
                         h2d_bytes_per_step=2 * 8 * mesh.n_n + 8 * conduct.size + 8 * mesh.n_e,
                         d2h_bytes_per_step=8 * mesh.n_n),
                gpu_launches=launches, clocks=clk, cpu_baseline=cpu)
    print(json.dumps(line))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if args.workload == "box":
            box_reference_arm(args, rank)
        elif args.workload == "seepage":
            if rank == 0:
                res = [seepage_cpu_seconds() for _ in range(max(1, min(args.steps, 3)))]
                n_full, n_sample = 220401, res[0][1]
                vals = [r[0] for r in res]
                v = sum(vals) / len(vals) * n_full / n_sample
                print(json.dumps(dict(metric=SEEPAGE_METRIC, value=v, unit="s/solve", n_gpus=args.gpus,
                                      steps=len(vals), warmup=0, ms_per_step=v * 1e3, higher_is_better=False,
                                      scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                                      impl="reference", config=dict(workload=SEEPAGE_WORKLOAD),
                                      cpu_baseline=dict(value=v, unit="s/solve", cores=1, kind="port",
                                                        sample=f"oracle seepage on the z = 1 m slice ({n_sample} "
                                                               "nodes) scaled by the node count"),
                                      e2e=dict(value=v, unit="s/solve", h2d_bytes_per_step=0,
                                               d2h_bytes_per_step=0))))
        elif args.workload == "ll":
            if rank == 0:
                print(json.dumps(dict(impl="reference", metric=LL_METRIC,
                                      unavailable="no CPU model of the limit-load step: the reference CPU path is "
                                                  "modelled for the SSR step workloads (hetero, ssr) and the box")))
        else:
            reference_arm(args, rank, world)
        return
    import datetime

    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local % max(torch.cuda.device_count(), 1))
    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", torch.cuda.current_device()))
    if args.workload in ("box", "ll", "seepage"):
        if args.workload == "box":
            run_box(args, rank)
        elif args.workload == "seepage":
            run_seepage(args, rank)
        else:
            run_ll(args, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    from slope_stability_octave_b200 import problems
    desc = WORKLOADS[args.workload][0]
    P = WORKLOADS[args.workload][1](problems).to_device()
    forms = {"all": ["plain", "mixed", "learned"], "both": ["plain", "mixed"]}.get(args.form, [args.form])
    out = {form: run_form(args, form, P, rank, world) for form in forms}
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    timed = {f: r for f, r in out.items() if r.get("timed")}
    if not timed:
        raise RuntimeError("no form was timed")
    head_form = next(f for f in ("learned", "mixed", "plain") if f in timed)
    head = timed[head_form]
    K = args.steps
    value_step = head["t_dev"] / K
    e2e_step = head["t_e2e"] / K
    peak, peak_kind = peaks()
    n_dof = P.dmesh.n_dof
    kbytes = kind_bytes(P, head["amg"], head["instr"][3], head["instr"][2])
    roofline = roofline_report(head, kbytes, K, peak, peak_kind, P.dmesh.n_blocks)
    base = timed["plain"] if "plain" in timed else head
    counts = step_counts(base)
    counts.update(n_int=P.dmesh.n_int, n_dof=n_dof)
    cpu = None
    if not args.no_cpu_baseline and args.gpus == 1:
        try:
            ratio, calib = cpu_calibration(args.workload, branch_mix=counts["branch_mix"])
            S, smp = cpu_sample(args.workload, branch_mix=counts["branch_mix"])
            v, _ = cpu_step_seconds(S, smp, counts, P.dmesh.n_int, n_dof)
            calib["model_full_step_s"] = round(v, 2)
            cpu = dict(value=v * ratio, unit=UNIT, cores=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                       kind="port", sample=cpu_sample_text(args.workload), calibration=calib)
        except Exception as exc:  # the CPU leg must not hide the GPU result
            cpu = dict(value=None, unit=UNIT, cores=None, kind="port", sample=f"failed: {exc}")
    h2d = 2 * 8 * n_dof
    d2h = 2 * 8 * n_dof
    forms_cfg = {}
    for form, r in out.items():
        if not r.get("timed"):
            forms_cfg[form] = dict(timed=False, init_s=round(r["t_init"], 2), network=r.get("learned"),
                                   note="the learned correction was rejected by its acceptance trial, so this "
                                        "form runs as the mixed form; its steps are not timed a second time")
            continue
        forms_cfg[form] = dict(
            s_per_step=r["t_dev"] / K, e2e_s_per_step=r["t_e2e"] / K, step_s=[round(t, 4) for t in r["step_s"]],
            device_allocs_in_timed_steps=r["alloc"],
            host_wall_and_cpu_s=[[round(a, 4), round(b, 4)] for a, b in r["host"]],
            continuation_steps=[s["step"] for s in r["steps"]],
            lambdas=r["lam"],
            newton_iterations=[s["newton_iterations_total"] for s in r["steps"]],
            linear_iterations=[s["linear_iterations"] for s in r["steps"]],
            attempts=[s["attempts"] for s in r["steps"]], deflation_basis=r["basis"], init_s=round(r["t_init"], 2),
            replay=r["replay"], gpu_launches=r["launches"],
            amg_levels=[(l["rows"], l["block"]) for l in r["amg"]["levels"]])
        if "learned" in r:
            forms_cfg[form]["network"] = r["learned"]
    for other in ("mixed", "learned"):
        if "plain" in timed and other in timed:
            # the two forms take the same continuation steps until their trajectories part
            # (near the limit load one form may need another Newton iteration and reach the
            # stop a step earlier): λ and time are compared over the longest common run of
            # identical step numbers, the whole-run ratio is kept beside it
            sp = [s["step"] for s in timed["plain"]["steps"]]
            so = [s["step"] for s in timed[other]["steps"]]
            m = 0
            while m < min(len(sp), len(so)) and sp[m] == so[m]:
                m += 1
            lp, lm = timed["plain"]["lam"], timed[other]["lam"]
            tp, to = timed["plain"]["step_s"], timed[other]["step_s"]
            forms_cfg[f"matched_steps_{other}_vs_plain"] = m
            forms_cfg[f"lambda_rel_err_{other}_vs_plain"] = (max(abs(a - b) / abs(a) for a, b in zip(lp[:m], lm[:m]))
                                                            if m else None)
            forms_cfg[f"speedup_{other}_vs_plain"] = (sum(tp[:m]) / sum(to[:m])) if m else None
            forms_cfg[f"speedup_{other}_vs_plain_whole_run"] = timed["plain"]["t_dev"] / timed[other]["t_dev"]
    line = dict(
        metric=METRIC, value=value_step, unit=UNIT, n_gpus=args.gpus, steps=K, warmup=args.warmup,
        ms_per_step=value_step * 1e3, higher_is_better=False, scaling="weak", vs_baseline=None,
        dtype={"plain": "f64", "mixed": "f64 (f32 V-cycle)", "learned": "f64 (f32 V-cycle, bf16 network)"}[head_form],
        data="synthetic (seeded mesh and material)",
        config=dict(workload=desc, form=head_form,
                    parallelism=f"replicas x{args.gpus}", solver="DFGMRES tol 1e-1 + AMG V-cycle, Newton tol 1e-4",
                    l2="working set > L2 (no flush needed)",
                    replay="state kept after the warm-up; when the continuation reaches its end the timed loop "
                           "restores it and continues with genuine accepted steps (forms.*.replay)",
                    forms=forms_cfg),
        e2e=dict(value=e2e_step, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h),
        gpu_launches=head["launches"],
        clocks=head["clocks"],
        roofline=roofline,
        cpu_baseline=cpu,
        counts=counts,
    )
    print(json.dumps(line))


if __name__ == "__main__":
    main()

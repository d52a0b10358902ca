"""Device mirror of the reference's LINEAR_SOLVERS package (DFGMRES with an AMG V-cycle).

  near_null_space_elasticity   +LINEAR_SOLVERS/near_null_space_elasticity_3D.m:1-108
                               (rigid-body modes on centred coordinates; 3 modes in 2D)
  AMG                          the BoomerAMG instance of hypre_boomeramg_mex.cpp
                               (setup_ijv / update_values / apply / clear), here a
                               smoothed-aggregation hierarchy built once per pattern
  DFGMRES                      +LINEAR_SOLVERS/DFGMRES.m:1-223 (deflation basis,
                               preconditioner hooks, copy semantics)
  set_linear_solver            +LINEAR_SOLVERS/set_linear_solver.m:1-71 (solver tokens)

Vectors are flat device tensors over all dim*n_n DOFs; Dirichlet DOFs carry zeros (the
block matrix has identity rows there), which leaves every inner product identical to the
reference's K(Q,Q) formulation.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import _lib
from .device import DeviceMesh, F64, cur_stream, hptr, matrix_generation, ptr


def near_null_space_elasticity(coord, Q=None, center=True):
    """Rigid-body modes (n_dof x nns, node-major rows), zero on Dirichlet DOFs when Q is given."""
    coord = np.asarray(coord, np.float64)
    dim, n_n = coord.shape
    X = coord - coord.mean(axis=1, keepdims=True) if center else coord
    if dim == 3:
        x, y, z = X
        modes = np.zeros((6, n_n, 3))
        modes[0, :, 0] = 1
        modes[1, :, 1] = 1
        modes[2, :, 2] = 1
        modes[3, :, 1], modes[3, :, 2] = -z, y
        modes[4, :, 0], modes[4, :, 2] = z, -x
        modes[5, :, 0], modes[5, :, 1] = -y, x
    else:
        x, y = X
        modes = np.zeros((3, n_n, 2))
        modes[0, :, 0] = 1
        modes[1, :, 1] = 1
        modes[2, :, 0], modes[2, :, 1] = -y, x
    Z = modes.reshape(modes.shape[0], -1).T.copy()          # (n_dof, nns), node-major rows
    if Q is not None:
        Z[~np.asarray(Q, bool).T.ravel()] = 0.0
    return Z


class AMG:
    """Device AMG preconditioner bound to a mesh's block pattern.

    The hierarchy's structure (aggregates on each level's strength graph) is built at the
    first value update, from those values, and reused for later updates, which redo only the
    numeric set-up on the device (the pattern is fixed per mesh)."""

    def __init__(self, dmesh: DeviceMesh, coord=None, mixed=False, max_levels=10, coarse_size=1200,
                 cheb_degree=3, cheb_ratio=10.0, power_its=10, theta=0.02, fine_half=False, symmetric=None):
        self.dmesh = dmesh
        coord = dmesh.mesh.coord if coord is None else coord
        if getattr(dmesh, "scalar", False):
            # scalar (pore-pressure) systems: the constant vector, zero on Dirichlet nodes
            Z = np.asarray(dmesh.mesh.Q, np.float64).reshape(-1, 1).copy()
        else:
            Z = near_null_space_elasticity(coord, dmesh.mesh.Q)
        self._nns = Z.shape[1]
        self._Z = np.ascontiguousarray(Z.T)                  # column-major n_dof x nns
        self._fixed = np.ascontiguousarray((~dmesh.mesh.Q.T.ravel()).astype(np.uint8))
        # the elasticity matrices K_r are symmetric (symmetrised in their assembly), so every
        # Galerkin matrix is formed on and above its diagonal and mirrored; the seepage
        # tangent is not symmetric (its E term) and takes the full product
        if symmetric is None:
            symmetric = not getattr(dmesh, "scalar", False)
        self.symmetric = bool(symmetric)
        self._opts = np.array([max_levels, coarse_size, cheb_degree, cheb_ratio, power_its, 1.0 if mixed else 0.0,
                               0.0, theta, 1.0 if (mixed and fine_half) else 0.0, 1.0 if symmetric else 0.0],
                              dtype=np.float64)
        self.handle = None
        self.setup_time = 0.0
        self.mixed = mixed
        self._A = None
        self._ready = None     # event after an update issued on a side stream

    def _create(self, K):
        h = C.c_void_p()
        t0 = time.perf_counter()
        _lib.call("sg_amg_create", self.dmesh.bsr, ptr(K), hptr(self._Z), self._nns, hptr(self._fixed),
                  hptr(self._opts), len(self._opts), C.byref(h), cur_stream())
        self.setup_time = time.perf_counter() - t0
        self.handle = h

    def __del__(self):
        c = getattr(self, "_clone", None)
        if c is not None and c.value:
            try:
                _lib.lib().sg_amg_destroy(c)
            except Exception:
                pass
            self._clone = None
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().sg_amg_destroy(h)
            except Exception:
                pass
            self.handle = None

    def update(self, K, stream=None):
        """Numeric set-up for the values K.  With ``stream`` (a side torch stream) the update is
        issued there after the work that produced K on the current stream, and the current
        stream waits for it only at the next ``wait`` (called by every consumer of the
        hierarchy), so the caller's independent work in between overlaps with it."""
        self.wait()
        self._A = K     # keep the values alive: the hierarchy references them
        if stream is None:
            if self.handle is None:
                self._create(K)
            _lib.call("sg_amg_update", self.handle, ptr(K), cur_stream())
            return
        produced = torch.cuda.Event()
        produced.record()
        stream.wait_event(produced)
        with torch.cuda.stream(stream):
            if self.handle is None:
                self._create(K)
            _lib.call("sg_amg_update", self.handle, ptr(K), cur_stream())
            self._ready = torch.cuda.Event()
            self._ready.record(stream)

    def wait(self):
        """Make the current stream wait for an update issued on a side stream."""
        if self._ready is not None:
            torch.cuda.current_stream().wait_event(self._ready)
            self._ready = None

    def apply(self, r, z):
        self.wait()
        _lib.call("sg_amg_apply", self.handle, ptr(r), ptr(z), cur_stream())

    def clone_handle(self):
        """Handle of a second set of cycle vectors over this hierarchy (created once, after
        the first update), for a V-cycle running beside this one on another stream."""
        if getattr(self, "_clone", None) is None:
            h = C.c_void_p()
            _lib.call("sg_amg_clone", self.handle, C.byref(h))
            self._clone = h
        return self._clone

    def info(self):
        buf = np.zeros(48, np.int64)
        _lib.call("sg_amg_info", self.handle, hptr(buf), 48)
        nl = int(buf[0])
        levels = [dict(block=int(buf[2 + 3 * i]), rows=int(buf[3 + 3 * i]), blocks=int(buf[4 + 3 * i]),
                       p_blocks=int(buf[32 + i])) for i in range(nl)]
        return dict(levels=levels, coarse_dense=int(buf[1]), mixed=bool(self.mixed),
                    cheb_degree=int(self._opts[2]))


class _Workspace:
    def __init__(self, n, maxit):
        h = C.c_void_p()
        _lib.call("sg_krylov_create", int(n), int(maxit), C.byref(h))
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().sg_krylov_destroy(h)
            except Exception:
                pass


class DFGMRES:
    """Deflated FGMRES with an AMG preconditioner (DFGMRES.m).  ``copy()`` shares the AMG
    instance and the Krylov workspace and copies the deflation basis, like the reference
    (copies share the closed-over HYPRE instance id, keep their own basis)."""

    def __init__(self, dmesh: DeviceMesh, tolerance, max_iterations, tolerance_deflation_basis, verbose=0,
                 amg: AMG | None = None, _ws=None, _pair=None):
        self.dmesh = dmesh
        self.tolerance = float(tolerance)
        self.max_iterations = int(max_iterations)
        self.tolerance_deflation_basis = float(tolerance_deflation_basis)
        self.verbose = verbose
        self.preconditioner = amg
        self.n = dmesh.n_dof
        self._ws = _ws if _ws is not None else _Workspace(self.n, self.max_iterations)
        # second Krylov workspace and stream for solve_pair (created on first use, shared by copies)
        self._pair = _pair if _pair is not None else {}
        self.basis = torch.empty((0, self.n), dtype=F64, device=dmesh.device)   # rows = columns of W
        # A W of the current basis and the matrix it was formed with ((data_ptr, generation)):
        # the solve uses it for the projection only while both still hold
        self.AW = None
        self._aw_key = None
        self.profiler = None
        self.last_iterations = 0
        self.last_relres = 0.0
        # optional learned node-wise correction of the V-cycle (learned.LearnedCorrection)
        self.learned = None
        self.overlap_update = True
        # solve_pair side by side: ~3-4 % less time per continuation step, but the two solves'
        # kernels then share the GPU, so per-kernel timings of a step are no longer those of a
        # kernel running alone; off unless asked for
        self.concurrent_pair = False
        # the projection of the deflated solve forms W'(A z) as (A W)' z, which needs a
        # symmetric A; False (the seepage tangent) makes the solve form A z instead
        self.symmetric_operator = True

    @property
    def k(self):
        return self.basis.shape[0]

    # the deflation basis lives in buffers whose row capacity is a multiple of 16, so that
    # appending a vector writes one row and copies of the basis fall into few allocation size
    # classes (the caching allocator then serves the Newton steps without new device memory)
    ROW_STEP = 16

    def _rows(self, k):
        if k == 0:
            return torch.empty((0, self.n), dtype=F64, device=self.dmesh.device)
        cap = -(-k // self.ROW_STEP) * self.ROW_STEP
        return torch.empty((cap, self.n), dtype=F64, device=self.dmesh.device)[:k]

    def _time(self, name, t0):
        if self.profiler is not None:
            torch.cuda.synchronize()
            self.profiler.add_time(name, time.perf_counter() - t0)

    def setup_preconditioner(self, K):
        """AMG numeric set-up for K.  When ``overlap_update`` is set (the default) it runs on
        the AMG's side stream: the Newton step's work up to the next solve (the residual at
        lambda + eps, the A-orthogonalisation of the deflation basis) overlaps with it, and
        the solve waits for it."""
        t0 = time.perf_counter()
        amg = self.preconditioner
        if amg is not None:
            if self.overlap_update and torch.cuda.is_available():
                if getattr(amg, "_side", None) is None:
                    amg._side = torch.cuda.Stream()
                amg.update(K, stream=amg._side)
            else:
                amg.update(K)
        self._time("DFGMRES.update_preconditioner", t0)

    # the reference's IJV hooks map onto the same update on the device pattern
    setup_preconditioner_ijv = setup_preconditioner
    update_preconditioner_values = setup_preconditioner

    def A_orthogonalize(self, K):
        t0 = time.perf_counter()
        k = self.k
        self.AW, self._aw_key = None, None
        if k > 0:
            B = self.basis.contiguous()
            AW = self._rows(k)
            kout = C.c_int32()
            _lib.call("sg_a_orthogonalize", self._ws.handle, self.dmesh.bsr, ptr(K), ptr(B), ptr(AW), k,
                      self.tolerance_deflation_basis, C.byref(kout), cur_stream())
            self.basis = B[: kout.value]
            self.AW = AW[: kout.value]
            self._aw_key = (K.data_ptr(), matrix_generation())
        self._time("DFGMRES.A_orthogonalize", t0)

    def solve(self, K, b):
        """x, nit = solve(K, b) on device vectors (dfgmres_solver.m)."""
        t0 = time.perf_counter()
        amg = self.preconditioner
        if amg is not None:
            amg.wait()
        lc = self.learned
        if lc is not None and amg is not None and lc.wants_training():
            # train on this system, then the acceptance trial: plain vs corrected solve of the
            # same system to the trial tolerance, timed on the device
            lc.train_on(amg, K, b)
            t1 = time.perf_counter()
            trial_tol = min(self.tolerance, lc.trial_tolerance)
            lc.off(amg)
            _, it_plain, _, t_plain = self._timed_solve(K, b, trial_tol)
            lc.features(K, b)
            lc.correction(amg)
            _, it_corr, rr_corr, t_corr = self._timed_solve(K, b, trial_tol)
            if not rr_corr <= trial_tol:
                it_corr, t_corr = self.max_iterations + 1, float("inf")
            lc.decide(it_plain, it_corr, time.perf_counter() - t1, t_plain=t_plain, t_corrected=t_corr)
        corrected = lc.before_solve(amg, K, b) if lc is not None else False
        x, nit, rr = self._solve_core(K, b)
        if corrected and not (rr <= self.tolerance):
            # the corrected preconditioner did not reach the tolerance: plain V-cycle
            self.learned.fallbacks += 1
            self.learned.off(amg)
            x, nit2, rr = self._solve_core(K, b)
            nit += nit2
        self.last_iterations = nit
        self.last_relres = rr
        self._time("DFGMRES.solve", t0)
        return x, nit

    def solve_pair(self, K, b1, b2):
        """(x1, nit1), (x2, nit2) = two independent solves with the same K and preconditioner
        (the W and V systems of newton_ind_SSR.m / newton_ind_LL.m).  With ``concurrent_pair``
        (and no learned correction in use: none, or trained and rejected) the second solve runs on its own
        stream, Krylov workspace and set of V-cycle vectors (an AMG clone) from a second host
        thread while the first runs here; the results equal two solves in sequence."""
        amg = self.preconditioner
        lc = self.learned
        idle_learned = lc is None or (lc.trained and not lc.enabled)   # no hook left to run
        if not (self.concurrent_pair and amg is not None and idle_learned and torch.cuda.is_available()):
            return self.solve(K, b1), self.solve(K, b2)
        if lc is not None:
            lc.solves += 2
        import threading
        t0 = time.perf_counter()
        amg.wait()
        pair = self._pair
        if "ws" not in pair:
            pair["ws"] = _Workspace(self.n, self.max_iterations)
            pair["stream"] = torch.cuda.Stream()
        clone = amg.clone_handle()
        side = pair["stream"]
        ready = torch.cuda.Event()
        ready.record()
        side.wait_event(ready)
        out = {}
        device = torch.cuda.current_device()

        def second():
            try:
                torch.cuda.set_device(device)
                with torch.cuda.stream(side):
                    out["r"] = self._solve_core(K, b2, ws=pair["ws"], M=clone)
            except BaseException as exc:  # re-raised in the calling thread
                out["e"] = exc

        th = threading.Thread(target=second)
        th.start()
        try:
            x1, it1, rr1 = self._solve_core(K, b1)
        finally:
            th.join()
        if "e" in out:
            raise out["e"]
        x2, it2, rr2 = out["r"]
        done = torch.cuda.Event()
        done.record(side)
        torch.cuda.current_stream().wait_event(done)
        x2.record_stream(torch.cuda.current_stream())   # allocated on the side stream, used here
        self.last_iterations, self.last_relres = it2, rr2
        self._time("DFGMRES.solve", t0)
        return (x1, it1), (x2, it2)

    def _timed_solve(self, K, b, tol):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x, it, rr = self._solve_core(K, b, tol)
        torch.cuda.synchronize()
        return x, it, rr, time.perf_counter() - t0

    def _solve_core(self, K, b, tol=None, ws=None, M=None):
        tol = self.tolerance if tol is None else tol
        ws = self._ws if ws is None else ws
        x = torch.empty_like(b)
        it = C.c_int32()
        rr = C.c_double()
        B = self.basis
        if self.preconditioner is not None:
            self.preconditioner.wait()
        if M is None:
            M = self.preconditioner.handle if self.preconditioner is not None else None
        aw_ok = (self.symmetric_operator and self.k > 0 and self.AW is not None
                 and self._aw_key == (K.data_ptr(), matrix_generation()))
        _lib.call("sg_dfgmres_solve", ws.handle, self.dmesh.bsr, ptr(K), M, ptr(B) if self.k else None,
                  ptr(self.AW) if aw_ok else None, self.k, ptr(b), ptr(x), tol, self.max_iterations,
                  C.byref(it), C.byref(rr), None, cur_stream())
        return x, it.value, rr.value

    def expand_deflation_basis(self, v):
        t0 = time.perf_counter()
        v = v.reshape(-1).to(F64)
        k = self.k
        base = self.basis._base
        if (base is not None and base.dim() == 2 and base.shape[0] > k and self.basis.is_contiguous()
                and self.basis.data_ptr() == base.data_ptr()):
            base[k].copy_(v)
            self.basis = base[: k + 1]
        else:
            nb = self._rows(k + 1)
            nb[:k].copy_(self.basis)
            nb[k].copy_(v)
            self.basis = nb
        self.AW, self._aw_key = None, None
        self._time("DFGMRES.expand_deflation_basis", t0)

    def copy(self):
        new = DFGMRES(self.dmesh, self.tolerance, self.max_iterations, self.tolerance_deflation_basis, self.verbose,
                      amg=self.preconditioner, _ws=self._ws, _pair=self._pair)
        new.concurrent_pair = self.concurrent_pair
        new.basis = new._rows(self.k)
        new.basis.copy_(self.basis)
        if self.AW is not None:
            new.AW, new._aw_key = self.AW.clone(), self._aw_key
        new.profiler = self.profiler
        new.learned = self.learned
        new.overlap_update = self.overlap_update
        new.symmetric_operator = self.symmetric_operator
        return new


def set_linear_solver(solver_type, linear_solver_tolerance, linear_solver_maxit, deflation_basis_tolerance,
                      linear_solver_printing, dmesh: DeviceMesh, coord=None, amg_opts=None, learned=None, cons=None):
    """Solver factory (set_linear_solver.m).  Tokens: 'DFGMRES_B200' (FP64 AMG V-cycle),
    'DFGMRES_B200_MIXED' (FP32 V-cycle inside the FP64 FGMRES; ``amg_opts`` fine_half=True
    makes its level-0 SpMVs read an FP16 copy of the matrix), 'DFGMRES_NONE' (no
    preconditioner).  ``learned`` (a dict of LearnedCorrection options, or True) adds the
    learned node-wise correction of the V-cycle; ``cons`` supplies its constitutive
    features (branch ids, reduced cohesion)."""
    tok = str(solver_type).upper()
    opts = dict(amg_opts or {})
    if tok in ("DFGMRES_B200", "DFGMRES_HYPRE_BOOMERAMG", "DFGMRES_BOOMERAMG", "BOOMERAMG", "HYPRE_BOOMERAMG"):
        amg = AMG(dmesh, coord, mixed=False, **opts)
    elif tok == "DFGMRES_B200_MIXED":
        amg = AMG(dmesh, coord, mixed=True, **opts)
    elif tok == "DFGMRES_NONE":
        amg = None
    else:
        raise ValueError(f"Bad choice of solver type: {solver_type}")
    solver = DFGMRES(dmesh, linear_solver_tolerance, linear_solver_maxit, deflation_basis_tolerance,
                     linear_solver_printing, amg=amg)
    if learned:
        from .learned import LearnedCorrection
        solver.learned = LearnedCorrection(dmesh, cons=cons, **(learned if isinstance(learned, dict) else {}))
    return solver

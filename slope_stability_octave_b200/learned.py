"""Learned node-wise correction of the AMG V-cycle inside DFGMRES.

No counterpart in the reference, whose DFGMRES (+LINEAR_SOLVERS/DFGMRES.m:134-147) is
preconditioned by one BoomerAMG V-cycle (hypre_boomeramg_mex.cpp:751-796).  With the
correction the preconditioner is

    z = V(r);   z += C (r - A z),   C_i = M_i G_i D_i^{-1}   (3 x 3 per node),

G_i = MLP(phi_i) from a per-node network (16 -> 64 -> 64 -> 9, ReLU; BF16 tensor-core
kernels with FP32 accumulation, written for sm_100a) over node features of the current
Newton system.  The network is trained on the GPU by the library's own forward and
backward kernels, on residual vectors that the plain preconditioner produces for the
Newton system it is solving, by minimising the true FP64 residual that the corrected
cycle leaves (optionally the energy norm of its error: A e = rz gives
|e - d|_A^2 - |e|_A^2 = d'A d - 2 d'rz, so no solve is needed).  The last layer starts at zero, so the untrained correction is exactly
the plain V-cycle, and ``DFGMRES.solve`` falls back to the plain V-cycle when a corrected
solve does not reach its tolerance.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import DeviceMesh, cur_stream, hptr, ptr

NPARAM = 6288


class LearnedCorrection:
    """Owner of the network, its training vectors and the correction handed to an AMG.

    train_at       index of the DFGMRES solve (0-based, counted over the solver's life)
                   whose Newton system provides the training vectors; training and the
                   acceptance trial happen just before that solve
    n_vectors      residual vectors collected for training
    steps, lr      full-batch Adam steps and learning rate
    loss           training objective: "residual" (the FP64 residual the corrected cycle
                   leaves) or "energy" (the energy norm of its error)
    trial_tolerance, trial_margin
                   the acceptance trial solves the training system plain and corrected to
                   min(solver tolerance, trial_tolerance) and keeps the correction only if it
                   needs fewer iterations and at most (1 - trial_margin) of the plain time
    """

    def __init__(self, dmesh: DeviceMesh, cons=None, train_at=0, n_vectors=12, steps=60, lr=3e-3, seed=0,
                 max_vectors=None, loss="residual", trial_tolerance=1e-6, trial_margin=0.05):
        if dmesh.dim != 3:
            raise ValueError("the learned correction is defined for 3D meshes")
        self.dmesh = dmesh
        self.cons = cons
        self.train_at = int(train_at)
        self.n_vectors = int(n_vectors)
        self.steps = int(steps)
        self.lr = float(lr)
        self.trial_tolerance = float(trial_tolerance)
        self.trial_margin = float(trial_margin)
        coord = np.ascontiguousarray(dmesh.mesh.coord, dtype=np.float64)   # 3 x n_n
        self._coord = np.ascontiguousarray(coord.T)                         # column-major 3 x n_n
        h = C.c_void_p()
        _lib.call("sg_learned_create", dmesh.handle, hptr(self._coord), int(max_vectors or max(self.n_vectors, 8)),
                  int(seed), C.byref(h))
        self.handle = h
        _lib.call("sg_learned_set_loss", h, {"residual": 0, "energy": 1}[loss])
        self.loss_kind = loss
        self.trained = False
        self.enabled = False
        self.gate = None
        self.solves = 0
        self.fallbacks = 0
        self.loss_hist = None
        self.train_seconds = 0.0

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().sg_learned_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------------ parameters
    def params(self):
        out = np.zeros(NPARAM, np.float32)
        _lib.call("sg_learned_params", self.handle, hptr(out), 0)
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == NPARAM
        _lib.call("sg_learned_params", self.handle, hptr(p), 1)

    # ------------------------------------------------------------------ per-system steps
    def features(self, K, residual):
        """Node features of the system K x = residual (device values on the mesh pattern)."""
        branch = c_bar = None
        if self.cons is not None:
            branch, c_bar = self.cons.branch, self.cons.c_bar
        _lib.call("sg_learned_features", self.handle, ptr(K), ptr(residual), ptr(branch) if branch is not None else None,
                  ptr(c_bar) if c_bar is not None else None, cur_stream())

    def correction(self, amg=None, out=None):
        """C from the current network (device n_n x 9 when ``out`` is given); set on ``amg``."""
        _lib.call("sg_learned_correction", self.handle, amg.handle if amg is not None else None,
                  ptr(out) if out is not None else None, cur_stream())

    def collect(self, amg, K, b, count, slot=0, append=False):
        _lib.call("sg_learned_collect", self.handle, amg.handle, self.dmesh.bsr, ptr(K), ptr(b), int(count), int(slot),
                  1 if append else 0, cur_stream())

    def loss(self, K, slot=0):
        out = C.c_double()
        _lib.call("sg_learned_loss", self.handle, self.dmesh.bsr, ptr(K), int(slot), C.byref(out), cur_stream())
        return out.value

    def gradient(self, K, slot=0):
        g = np.zeros(NPARAM, np.float32)
        loss = C.c_double()
        _lib.call("sg_learned_gradient", self.handle, self.dmesh.bsr, ptr(K), int(slot), hptr(g), C.byref(loss),
                  cur_stream())
        return g, loss.value

    def train(self, K, steps=None, lr=None):
        steps = self.steps if steps is None else int(steps)
        hist = np.zeros(max(steps, 1))
        _lib.call("sg_learned_train", self.handle, self.dmesh.bsr, ptr(K), steps, float(self.lr if lr is None else lr),
                  hptr(hist), cur_stream())
        self.loss_hist = hist[:steps]
        return self.loss_hist

    def export(self, what, index=0):
        """Host copy of internal state: 'features' (n_pad x 16 float32 BF16 values), 'G',
        'Dinv' (n_n x 3 x 3), 'rz0' / 'rz1' (residual vector ``index`` of slot 0 / 1), 'C'."""
        nn, n_pad = self.dmesh.n_n, self.info()["n_pad"]
        if what == "features":
            bits = np.zeros((n_pad, 16), np.uint16)
            _lib.call("sg_learned_export", self.handle, 0, 0, hptr(bits))
            return (bits.astype(np.uint32) << 16).view(np.float32)
        if what == "G":
            out = np.zeros((n_pad, 16), np.float32)
            _lib.call("sg_learned_export", self.handle, 1, 0, hptr(out))
            return out
        if what in ("Dinv", "C"):
            out = np.zeros((nn, 3, 3))
            _lib.call("sg_learned_export", self.handle, 2 if what == "Dinv" else 5, 0, hptr(out))
            return out
        if what in ("rz0", "rz1"):
            out = np.zeros(self.dmesh.n_dof)
            _lib.call("sg_learned_export", self.handle, 3 if what == "rz0" else 4, int(index), hptr(out))
            return out
        raise ValueError(what)

    def info(self):
        buf = np.zeros(5, np.int64)
        _lib.call("sg_learned_info", self.handle, hptr(buf))
        return dict(nparam=int(buf[0]), vectors=int(buf[1]), held_out=int(buf[2]), n_pad=int(buf[3]),
                    adam_steps=int(buf[4]))

    # ------------------------------------------------------------------ DFGMRES hook
    def wants_training(self):
        return not self.trained and self.solves >= self.train_at

    def train_on(self, amg, K, b):
        """Collect this system's residual vectors and train (called by DFGMRES.solve)."""
        import time
        t0 = time.perf_counter()
        self.features(K, b)
        self.collect(amg, K, b, self.n_vectors, slot=0)
        self.train(K)
        torch.cuda.synchronize()
        self.train_seconds += time.perf_counter() - t0
        self.trained = True

    def decide(self, it_plain, it_corrected, seconds=0.0, t_plain=None, t_corrected=None):
        """Acceptance gate: keep the correction only if the trial solve of the training system
        (to the trial tolerance) needed fewer DFGMRES iterations with it than without and, when
        the trial was timed, took at most (1 - trial_margin) of the plain solve's time: the
        correction costs an extra fine-level SpMV per iteration, so fewer iterations alone do
        not make it faster."""
        faster = t_plain is None or t_corrected is None or t_corrected <= (1.0 - self.trial_margin) * t_plain
        self.gate = dict(plain_iterations=int(it_plain), corrected_iterations=int(it_corrected),
                         accepted=bool(it_corrected < it_plain and faster))
        if t_plain is not None:
            self.gate.update(plain_s=round(float(t_plain), 4), corrected_s=round(float(t_corrected), 4),
                             tolerance=self.trial_tolerance)
        self.enabled = self.gate["accepted"]
        self.train_seconds += seconds

    def before_solve(self, amg, K, b):
        """Set the correction for the system K x = b on the AMG instance when the network is
        trained and accepted; otherwise switch it off.  True when the solve runs corrected."""
        self.solves += 1
        if amg is None:
            return False
        if not (self.trained and self.enabled):
            self.off(amg)
            return False
        self.features(K, b)
        self.correction(amg)
        return True

    def off(self, amg):
        if amg is not None:
            _lib.call("sg_amg_set_correction", amg.handle, None, cur_stream())

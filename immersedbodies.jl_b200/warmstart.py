"""Learned CG warm start for moving bodies.

The reference solves the force system B F~b = Ftmp of a moving body with plain
conjugate gradients started from the previous step's F~b (src/coupling.jl:194-202).
Installed on a solver (`GpuCnabSolver.set_warm_start`), the learned start takes
two Galerkin steps in the B-energy norm before the CG: one along the last change
of the solution (the extrapolated guess x_e), one along a correction that
`WarmStartNet`, a small 1D convolutional network over the body points, computes
from x_e's residual b - B x_e.  The CG still runs to the configured tolerance, so
only the number of iterations changes.

Everything the network computes -- forward, backward, loss, Adam -- runs in the
library's own CUDA kernels (csrc/warmstart.cu).  Training data comes from the
solver itself: `collect_samples` steps a solver in the extrapolated mode and
records, per step, the ten feature channels of every body point and the error
of the extrapolated guess.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _abi

FEATURES = 10  # residual of x_e x/y, F1 x/y, F1 - F2 x/y, ub x/y, cos/sin of the body angle
OUTPUTS = 2    # the error of the extrapolated guess, F~b - x_e, x and y (in units of the residual's RMS)


class WarmStartNet:
    """1D convolutional network on one device: `layers` convolutions of odd
    width `kernel` with zero padding, `width` channels between them, tanh after
    every layer but the last; per-channel input and output normalisation."""

    def __init__(self, *, width: int = 64, kernel: int = 5, layers: int = 4, seed: int = 2026, device: int = 0,
                 cin: int = FEATURES, cout: int = OUTPUTS):
        self.lib = _abi.load()
        self.arch = dict(width=width, kernel=kernel, layers=layers, cin=cin, cout=cout)
        self._h = C.c_void_p()
        rc = self.lib.ibpm_net_create(cin, width, kernel, layers, cout, seed, device, C.byref(self._h))
        if rc != _abi.IBPM_OK:
            raise _abi.IbpmError(rc, self.lib.ibpm_net_last_error(None).decode())
        self.cin, self.cout = cin, cout

    def _check(self, rc: int):
        if rc < 0:
            raise _abi.IbpmError(rc, self.lib.ibpm_net_last_error(self._h).decode())
        return rc

    def close(self):
        if self._h:
            self.lib.ibpm_net_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def num_params(self) -> int:
        return int(self.lib.ibpm_net_num_params(self._h))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.num_params, dtype=np.float32)
        self._check(self.lib.ibpm_net_get_params(self._h, _abi.fptr(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        self._check(self.lib.ibpm_net_set_params(self._h, _abi.fptr(p)))

    def set_normalisation(self, in_mean, in_std, out_mean, out_std):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (in_mean, in_std, out_mean, out_std)]
        self._check(self.lib.ibpm_net_set_normalisation(self._h, *[_abi.fptr(v) for v in a]))

    def normalisation(self):
        a = [np.empty(n, dtype=np.float32) for n in (self.cin, self.cin, self.cout, self.cout)]
        self._check(self.lib.ibpm_net_get_normalisation(self._h, *[_abi.fptr(v) for v in a]))
        return tuple(a)

    def fit_normalisation(self, x: np.ndarray, t: np.ndarray, floor: float = 1e-6):
        """Per-channel mean and standard deviation of samples x [S][cin][n] and
        targets t [S][cout][n] (standard deviations floored at `floor` times the
        largest one, and at 1 for a constant channel)."""
        def stats(a):
            m = a.mean(axis=(0, 2))
            s = a.std(axis=(0, 2))
            top = s.max() if s.size and s.max() > 0 else 1.0
            s = np.where(s > floor * top, s, np.where(top > 0, floor * top, 1.0))
            s = np.where(s > 0, s, 1.0)
            return m, s
        im, isd = stats(np.asarray(x, dtype=np.float64))
        om, osd = stats(np.asarray(t, dtype=np.float64))
        self.set_normalisation(im, isd, om, osd)

    def forward(self, x: np.ndarray) -> np.ndarray:
        """Predictions (solver units) for raw samples x [B][cin][n]."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        B, _, n = x.shape
        y = np.empty((B, self.cout, n), dtype=np.float32)
        self._check(self.lib.ibpm_net_forward(self._h, _abi.fptr(x), B, n, _abi.fptr(y)))
        return y

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        """(loss, gradient) on normalised targets: the squared error plus that of
        its running sum along the body points (which weighs smooth errors more)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        g = np.empty(self.num_params, dtype=np.float32)
        self._check(self.lib.ibpm_net_loss_grad(self._h, _abi.fptr(x), _abi.fptr(t), x.shape[0], x.shape[2],
                                                _abi.fptr(loss), _abi.fptr(g)))
        return float(loss[0]), g

    def train(self, x: np.ndarray, t: np.ndarray, *, epochs: int = 100, batch: int = 64, lr: float = 1e-3,
              seed: int = 7) -> np.ndarray:
        """Adam on shuffled full batches; returns the mean batch loss per epoch."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        self._check(self.lib.ibpm_net_train(self._h, _abi.fptr(x), _abi.fptr(t), x.shape[0], x.shape[2], epochs,
                                            batch, lr, seed, _abi.fptr(losses)))
        return losses

    def save(self, path: str):
        im, isd, om, osd = self.normalisation()
        np.savez(path, params=self.get_params(), in_mean=im, in_std=isd, out_mean=om, out_std=osd,
                 **{k: np.int64(v) for k, v in self.arch.items()})

    @classmethod
    def load(cls, path: str, device: int = 0) -> "WarmStartNet":
        d = np.load(path)
        net = cls(width=int(d["width"]), kernel=int(d["kernel"]), layers=int(d["layers"]), cin=int(d["cin"]),
                  cout=int(d["cout"]), device=device)
        net.set_params(d["params"])
        net.set_normalisation(d["in_mean"], d["in_std"], d["out_mean"], d["out_std"])
        return net


def collect_samples(solver, nsteps: int, skip: int = 0):
    """Steps `solver` skip + nsteps times in the extrapolated mode and returns
    the warm-start samples of the last nsteps steps: features [nsteps][10][np],
    targets [nsteps][2][np] and the CG iteration count of every step."""
    solver.set_warm_start(None, mode="extrapolated")
    for _ in range(skip):
        solver.advance_()
    X, T, iters = [], [], []
    for _ in range(nsteps):
        solver.advance_()
        f, t = solver.warm_start_sample()
        X.append(f)
        T.append(t)
        iters.append(solver.info().last_cg_iters)
    return np.stack(X), np.stack(T), np.asarray(iters)


def cg_iterations(solver, nsteps: int) -> np.ndarray:
    """CG iterations of each of the next nsteps steps."""
    out = []
    for _ in range(nsteps):
        solver.advance_()
        out.append(solver.info().last_cg_iters)
    return np.asarray(out)


def make_training_set(make_solver, ks: Sequence[float], nsteps: int, skip: int = 0):
    """Concatenated samples of one solver per reduced frequency k in ks."""
    xs, ts = [], []
    for k in ks:
        s = make_solver(k)
        x, t, _ = collect_samples(s, nsteps, skip)
        xs.append(x)
        ts.append(t)
        del s
    return np.concatenate(xs), np.concatenate(ts)

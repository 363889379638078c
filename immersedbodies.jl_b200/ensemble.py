"""Ensembles of independent cases stepped together on one GPU.

The reference steps one case per solver.  A single small case (a few hundred
cells a side, three levels) fills only a few percent of a B200, so an ensemble
enqueues every case's step on that case's own stream before waiting for any
(`ibpm_ensemble_advance`); the cases' step graphs then run side by side.  Each
case's results are exactly those of stepping it alone.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _abi
from .problem import set_time_index_, timestep


class Ensemble:
    """Independent `GpuCnabSolver`s (any sizes, bodies and precisions) stepped together."""

    def __init__(self, solvers: Sequence):
        self.solvers = list(solvers)
        self.lib = _abi.load()
        self._h = C.c_void_p()
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        rc = self.lib.ibpm_ensemble_create(arr, len(self.solvers), C.byref(self._h))
        if rc != _abi.IBPM_OK:
            raise _abi.IbpmError(rc, "ibpm_ensemble_create failed")

    def close(self):
        if self._h:
            self.lib.ibpm_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance_(self, nsteps: int = 1, fetch_forces: bool = True):
        """advance! every case nsteps times; with fetch_forces each case's
        state.fb is read back afterwards (as GpuCnabSolver.advance_ does)."""
        n = len(self.solvers)
        params = (_abi.ibpm_step_params * (nsteps * n))()
        keep = []
        for k in range(nsteps):
            for c, s in enumerate(self.solvers):
                st = s.state
                p = s.step_params(st.t0 + timestep(st.prob) * (st.index + k))
                q = params[k * n + c]
                q.freestream[0], q.freestream[1] = p.freestream[0], p.freestream[1]
                for j in range(6):
                    q.grid_motion[j] = p.grid_motion[j]
                if p.body_motion:
                    m = s._motion.copy()
                    keep.append(m)
                    q.body_motion = m.ctypes.data_as(_abi._dp)
        rc = self.lib.ibpm_ensemble_advance(self._h, nsteps, params)
        if rc < 0:
            raise _abi.IbpmError(rc, self.lib.ibpm_ensemble_last_error(self._h).decode())
        for s in self.solvers:
            st = s.state
            set_time_index_(st, st.index + nsteps)
            s._stale = True
            if fetch_forces:
                _abi.check(s.lib, s._h, s.lib.ibpm_get_forces(s._h, _abi.dptr(st.fb), None))
        return rc

    def total_forces(self) -> np.ndarray:
        """boundary_total_force of every case (n x 2)."""
        return np.stack([s.total_force() for s in self.solvers])

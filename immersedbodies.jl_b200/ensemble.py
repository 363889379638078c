"""Ensembles of independent cases stepped together on one GPU.

The reference steps one case per solver.  A single small case (a few hundred
cells a side, three levels) fills only a few percent of a B200.  An ensemble
(`ibpm_ensemble_advance`) therefore batches its static-body cases of one shape
(precision, nx, ny, levels, grid step, time step): their fields are stacked and
each line pass, nonlinear term, curl and coupling kernel runs once over all of
them, one CUDA graph per group step; the rest step side by side on their own
streams.  Each case's results are exactly those of stepping it alone.
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

    def groups(self):
        """(number of batched groups, number of cases they hold)."""
        ng, nb = C.c_int32(), C.c_int32()
        self.lib.ibpm_ensemble_groups(self._h, C.byref(ng), C.byref(nb))
        return ng.value, nb.value

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


def case_cost(prob) -> int:
    """Work of one step of a case, in grid points: every level of the nested
    grid has the finest level's nx x ny points."""
    g = prob.grid
    return int(g.base.n[0]) * int(g.base.n[1]) * int(g.nlevel)


def shard_cases(costs: Sequence[int], world: int) -> list:
    """Partitions cases 0..n-1 over `world` ranks, balanced by cost: the cases
    are taken in order of decreasing cost (ties by index) and each goes to the
    rank with the least cost so far (ties by rank).  Deterministic, so every
    rank computes the same partition without communicating.  Returns one sorted
    list of case indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-int(costs[k]), k))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += int(costs[k])
    return [sorted(p) for p in parts]


def gather_case_forces(n_cases: int, local_ids: Sequence[int], local_forces, pg=None, device="cpu") -> np.ndarray:
    """Per-case total forces of a sharded ensemble, on every rank: each rank
    contributes the rows of its own cases (n_local x 2) and the rest as zeros,
    and one sum all-reduce over ranks fills the n_cases x 2 table (every row has
    exactly one contributor, so the sum is exact).  A third column counts the
    contributors of each row; a row that is not 1 (a case that no rank or two
    ranks stepped) raises ValueError.  pg is torch.distributed (or None for one
    process); device holds the reduction buffer ("cpu" under gloo, "cuda" under
    NCCL)."""
    import torch

    t = torch.zeros((n_cases, 3), dtype=torch.float64, device=device)
    lf = np.asarray(local_forces, dtype=np.float64).reshape(-1, 2)
    ids = list(local_ids)
    if len(ids) != lf.shape[0]:
        raise ValueError("one force row per local case is required")
    if ids:
        idx = torch.as_tensor(ids, dtype=torch.long, device=device)
        t[idx, 0:2] = torch.as_tensor(lf, dtype=torch.float64, device=device)
        t[idx, 2] = 1.0
    if pg is not None:
        pg.all_reduce(t, op=pg.ReduceOp.SUM)
    out = t.cpu().numpy()
    if not np.all(out[:, 2] == 1.0):
        bad = np.nonzero(out[:, 2] != 1.0)[0][:8].tolist()
        raise ValueError(f"cases without exactly one owning rank: {bad}")
    return out[:, :2].copy()

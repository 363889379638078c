"""Solver interface, mirroring ImmersedBodies.jl's `src/solver.jl`.

`GpuCnabSolver` is the drop-in for `CnabSolver` (solver.jl:84-190): the same
`create_solver` / `advance_` / `getstate` / `solve` / `solve_` entry points,
with every step computed by libibpm_b200.so on the GPU.  Host callbacks
(freestream_vel(t), body motion(t), grid motion(t)) are evaluated here and
pushed to the device as per-step scalars.  The host `State` is synchronised
lazily: index, t and fb after every step; full fields on `getstate`.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

import numpy as np

from . import _abi
from .problem import (MovingRigidBody, Problem, State, StaticBody, inc_time_index_, set_time_index_, timestep,
                      update_vars_)


class AbstractSolver:
    """abstract type AbstractSolver (solver.jl:6)."""

    def advance_(self):
        raise NotImplementedError

    def getstate(self) -> State:
        raise NotImplementedError


def _init_static_panels(state: State):
    """_init_body_motion!'s effect on the panels of static bodies (bodies.jl:1-6, 33-41)."""
    for _, body, r in state.prob.bodies.preset:
        if isinstance(body, StaticBody):
            state.panels.xb[r.start:r.stop, :] = body.panels.xb
            state.panels.ds[r.start:r.stop] = body.panels.ds
            state.panels.ub[r.start:r.stop, :] = 0.0


class GpuCnabSolver(AbstractSolver):
    """CnabSolver(state; cg=(maxiter, reltol, abstol)) on the GPU.

    precision="fp64" is the plain drop-in path; precision="fp32" keeps every
    level's fields and transforms in FP32 (FP64 scans, boundary values, CG,
    force sums and B^-1); precision="mixed" keeps level 1, the body's level, in
    FP64 and the coarser levels in FP32 (static bodies)."""

    def __init__(self, state: State, *, cg: Optional[dict] = None, device: int = 0, precision: str = "fp64"):
        self.lib = _abi.load()
        self.state = state
        prob = state.prob
        self._h = C.c_void_p()
        bodies = prob.bodies
        kinds = np.array([b.kind for _, b, _ in bodies.preset], dtype=np.int32)
        starts = np.array([r.start for _, _, r in bodies.preset] + [bodies.npanel], dtype=np.int32)
        xb = np.asfortranarray(np.vstack([b.panels.xb for _, b, _ in bodies.preset]))
        ds = np.concatenate([b.panels.ds for _, b, _ in bodies.preset])
        self._keep = (kinds, starts, xb, ds)
        g = prob.grid
        p = _abi.ibpm_problem(
            nx=g.base.n[0], ny=g.base.n[1], nlevel=g.nlevel, h=g.base.h, x0=g.base.x0[0], y0=g.base.x0[1],
            Re=prob.fluid.Re, dt=timestep(prob), npanel=bodies.npanel, nbody=len(kinds),
            body_kind=kinds.ctypes.data_as(_abi._ip), body_start=starts.ctypes.data_as(_abi._ip),
            body_xb=_abi.dptr(xb), body_ds=_abi.dptr(ds), grid_moving=1 if prob.fluid.grid_motion.moving else 0)
        opt = _abi.ibpm_options()
        self.lib.ibpm_default_options(C.byref(opt))
        opt.device = device
        opt.precision = {"fp64": _abi.IBPM_FP64, "fp32": _abi.IBPM_FP32, "mixed": _abi.IBPM_MIXED_L1}[precision]
        self.precision = precision
        for k, v in (cg or {}).items():
            setattr(opt, {"maxiter": "cg_maxiter", "reltol": "cg_reltol", "abstol": "cg_abstol"}[k], v)
        rc = self.lib.ibpm_create(C.byref(p), C.byref(opt), C.byref(self._h))
        if rc != _abi.IBPM_OK:
            raise _abi.IbpmError(rc, self.lib.ibpm_last_error(None).decode())
        _init_static_panels(state)
        self._upload(state)
        self._moving = [isinstance(b, MovingRigidBody) for _, b, _ in bodies.preset]
        self._motion = np.zeros((len(kinds), 6))
        self._params = _abi.ibpm_step_params()
        self._stale = False
        self.last_status = 0

    def close(self):
        """Frees the device state now (also done when the solver is collected).
        An ensemble holding this solver then refuses to advance."""
        h = getattr(self, "_h", None)
        if h:
            self.lib.ibpm_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def _view(self, s: State) -> _abi.ibpm_state_view:
        v = _abi.ibpm_state_view()
        v.index = s.index
        v.t0 = s.t0
        v.q, v.q0, v.gamma, v.psi = (_abi.dptr(s.q), _abi.dptr(s.q0), _abi.dptr(s.Gamma), _abi.dptr(s.psi))
        v.nonlin1, v.nonlin2 = _abi.dptr(s.nonlin[0]), _abi.dptr(s.nonlin[1])
        v.xb, v.ds, v.ub, v.fbt = (_abi.dptr(s.panels.xb), _abi.dptr(s.panels.ds), _abi.dptr(s.panels.ub),
                                   _abi.dptr(s.Fbt))
        v.freestream[0], v.freestream[1] = s.freestream_vel
        return v

    def _upload(self, s: State):
        _abi.check(self.lib, self._h, self.lib.ibpm_set_state(self._h, C.byref(self._view(s))))

    def sync(self) -> State:
        """Copy the full device state into the host State."""
        s = self.state
        v = self._view(s)
        _abi.check(self.lib, self._h, self.lib.ibpm_get_state(self._h, C.byref(v)))
        s.freestream_vel = (v.freestream[0], v.freestream[1])
        update_vars_(s)
        self._stale = False
        return s

    def getstate(self) -> State:
        return self.sync() if self._stale else self.state

    def step_params(self, t: float) -> _abi.ibpm_step_params:
        """The host callbacks' values at time t, as one ibpm_step_params."""
        prob = self.state.prob
        prm = self._params
        fs = prob.fluid.freestream_vel(t)
        prm.freestream[0], prm.freestream[1] = float(fs[0]), float(fs[1])
        gm = prob.fluid.grid_motion
        row = gm(t).as_row() if gm.moving else [0.0] * 6
        for k in range(6):
            prm.grid_motion[k] = row[k]
        if any(self._moving):
            for b, (_, body, _) in enumerate(prob.bodies.preset):
                if self._moving[b]:
                    self._motion[b] = body.motion(t).as_row()
            prm.body_motion = self._motion.ctypes.data_as(_abi._dp)
        else:
            prm.body_motion = None
        return prm

    def advance_(self):
        """advance!(solver) (solver.jl:155-190)."""
        s = self.state
        inc_time_index_(s)
        prm = self.step_params(s.t)
        s.freestream_vel = (prm.freestream[0], prm.freestream[1])
        rc = self.lib.ibpm_advance(self._h, 1, C.byref(prm))
        if rc < 0:
            set_time_index_(s, s.index - 1)
        self.last_status = _abi.check(self.lib, self._h, rc)
        _abi.check(self.lib, self._h, self.lib.ibpm_get_forces(self._h, _abi.dptr(s.fb), None))
        self._stale = True

    def _field(self, field: int, level: int, shape) -> np.ndarray:
        out = np.empty(shape, order="F")
        _abi.check(self.lib, self._h, self.lib.ibpm_get_field(self._h, field, level, _abi.dptr(out)))
        return out

    def vorticity(self, level: int = 1) -> np.ndarray:
        """vorticity! of one level (1-based), computed on the device: Γ / hc², (nx-1) x (ny-1)."""
        nx, ny = self.state.prob.grid.base.n
        return self._field(0, level, (nx - 1, ny - 1))

    def x_velocity(self, level: int = 1) -> np.ndarray:
        """x_velocity! of one level, computed on the device: (q + q0)_u / hc, (nx+1) x ny."""
        nx, ny = self.state.prob.grid.base.n
        return self._field(1, level, (nx + 1, ny))

    def y_velocity(self, level: int = 1) -> np.ndarray:
        """y_velocity! of one level, computed on the device: (q + q0)_v / hc, nx x (ny+1)."""
        nx, ny = self.state.prob.grid.base.n
        return self._field(2, level, (nx, ny + 1))

    def total_force(self) -> np.ndarray:
        out = np.zeros(2)
        _abi.check(self.lib, self._h, self.lib.ibpm_get_forces(self._h, None, _abi.dptr(out)))
        return out

    def info(self) -> _abi.ibpm_info:
        i = _abi.ibpm_info()
        _abi.check(self.lib, self._h, self.lib.ibpm_get_info(self._h, C.byref(i)))
        return i

    def kernel_launches(self) -> int:
        return int(self.lib.ibpm_kernel_launches(self._h))

    def stream_handle(self) -> int:
        """The library's cudaStream_t, as an integer (for CUDA-event timing on it)."""
        return int(self.lib.ibpm_stream(self._h) or 0)

    def profile(self, enable: bool):
        _abi.check(self.lib, self._h, self.lib.ibpm_profile(self._h, 1 if enable else 0))

    def profile_read(self, kclass: str):
        """(launches, device ms, algorithmic bytes) of one kernel class since profile(True)."""
        n, ms, b = C.c_int64(), C.c_double(), C.c_double()
        _abi.check(self.lib, self._h, self.lib.ibpm_profile_read(self._h, _abi.KCLASS[kclass], C.byref(n),
                                                                  C.byref(ms), C.byref(b)))
        return n.value, ms.value, b.value

    def diag_solve(self, op: int, level: int, b: np.ndarray) -> np.ndarray:
        """One DST-diagonalised solve on the device: op 0 Δinv, 1 A, 2 Ainv (at
        `level`); op 3..5 the same with the tensor-core transforms of one BF16
        product, 6..8 with three (split BF16)."""
        b = np.asfortranarray(b, dtype=np.float64)
        x = np.empty_like(b, order="F")
        _abi.check(self.lib, self._h, self.lib.ibpm_diag_solve(self._h, op, level, _abi.dptr(b), _abi.dptr(x)))
        return x

    def diag_apply_B(self, z: np.ndarray) -> np.ndarray:
        z = np.ascontiguousarray(z, dtype=np.float64)
        x = np.empty_like(z)
        _abi.check(self.lib, self._h, self.lib.ibpm_diag_apply_B(self._h, _abi.dptr(z), _abi.dptr(x)))
        return x

    def diag_binv(self) -> np.ndarray:
        n = 2 * self.state.prob.bodies.npanel
        out = np.empty((n, n), order="F")
        _abi.check(self.lib, self._h, self.lib.ibpm_diag_binv(self._h, _abi.dptr(out)))
        return out

    def diag_vort2flux(self, gamma: np.ndarray):
        """vort2flux on the device: returns (coarsified gamma, psi, q)."""
        g = np.asfortranarray(gamma, dtype=np.float64).copy(order="F")
        psi = np.zeros_like(g, order="F")
        q = np.zeros((self.state.q.shape[0], g.shape[1]), order="F")
        _abi.check(self.lib, self._h, self.lib.ibpm_diag_vort2flux(self._h, _abi.dptr(g), _abi.dptr(psi),
                                                                    _abi.dptr(q)))
        return g, psi, q

    def diag_reg_rot(self, f: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros(self.state.Gamma.shape[0])
        _abi.check(self.lib, self._h, self.lib.ibpm_diag_reg(self._h, _abi.dptr(f), _abi.dptr(out), None, None))
        return out

    def diag_regT(self, q1: np.ndarray) -> np.ndarray:
        q1 = np.ascontiguousarray(q1, dtype=np.float64)
        out = np.zeros(2 * self.state.prob.bodies.npanel)
        _abi.check(self.lib, self._h, self.lib.ibpm_diag_reg(self._h, None, None, _abi.dptr(q1), _abi.dptr(out)))
        return out

    def set_warm_start(self, net=None, mode: Optional[str] = None, depth: int = 8):
        """CG initial guess of this moving-body solver: "previous" (the reference's
        start from the previous F~b), "extrapolated" (Galerkin step along the last
        change F1 - F2), "learned" (then along a `WarmStartNet`'s correction; the
        default when net is given), "projected" (Galerkin over the last `depth`
        solutions), "direct" (B^-1 b, B assembled and inverted on the GPU every
        `depth` steps; FP64 only) or "preconditioned" (as "direct", and CG
        preconditioned by that inverse: a few iterations between rebuilds; not the
        reference's unpreconditioned iteration) or "preconditioned_extrapolated"
        (as "preconditioned", started from B^-1 b plus the stale error
        F - B^-1 b extrapolated from the last steps).  Keep the network alive
        while it is installed."""
        mode = mode or ("learned" if net is not None else "previous")
        m = {"previous": _abi.IBPM_WS_PREVIOUS, "learned": _abi.IBPM_WS_LEARNED,
             "extrapolated": _abi.IBPM_WS_EXTRAPOLATED, "projected": _abi.IBPM_WS_PROJECTED,
             "direct": _abi.IBPM_WS_DIRECT, "preconditioned": _abi.IBPM_WS_PRECONDITIONED,
             "preconditioned_extrapolated": _abi.IBPM_WS_PRECOND_EXTRAP}[mode]
        _abi.check(self.lib, self._h, self.lib.ibpm_set_warm_start(self._h, m, net.handle if net is not None else None,
                                                                    depth))
        self._warm_net = net

    def set_rebuild_transform(self, products: int):
        """How the preconditioned modes assemble the B they invert: 0 with the
        step's FP64 transforms, 1 or 3 with dense DST-I passes on the tensor
        cores (one BF16 product, or three on split BF16 operands).  CG runs to
        the same tolerance either way."""
        _abi.check(self.lib, self._h, self.lib.ibpm_set_rebuild_transform(self._h, int(products)))

    def warm_start_sample(self, prediction: bool = False):
        """(features [10][np], target [2][np]) of the last step: the warm start's
        inputs and the error of its extrapolated guess (converged F~b - x_e); with
        prediction=True also the network's correction as the step used it."""
        n = self.state.prob.bodies.npanel
        f = np.empty((10, n), dtype=np.float32)
        t = np.empty((2, n), dtype=np.float32)
        p = np.empty((2, n), dtype=np.float32) if prediction else None
        _abi.check(self.lib, self._h, self.lib.ibpm_warm_start_sample(self._h, _abi.fptr(f), _abi.fptr(t),
                                                                       _abi.fptr(p)))
        return (f, t, p) if prediction else (f, t)

    def advance_many(self, nsteps: int):
        """nsteps advance! calls in one library call (params evaluated on the host
        up front); the host State's index/t/fb are updated at the end."""
        s = self.state
        arr = (_abi.ibpm_step_params * nsteps)()
        motions = []
        for k in range(nsteps):
            t = s.t0 + timestep(s.prob) * (s.index + k)
            p = self.step_params(t)
            arr[k].freestream[0], arr[k].freestream[1] = p.freestream[0], p.freestream[1]
            for j in range(6):
                arr[k].grid_motion[j] = p.grid_motion[j]
            if p.body_motion:
                m = self._motion.copy()
                motions.append(m)
                arr[k].body_motion = m.ctypes.data_as(_abi._dp)
        rc = self.lib.ibpm_advance(self._h, nsteps, arr)
        self.last_status = _abi.check(self.lib, self._h, rc)
        set_time_index_(s, s.index + nsteps)
        s.freestream_vel = (arr[nsteps - 1].freestream[0], arr[nsteps - 1].freestream[1]) if nsteps else s.freestream_vel
        _abi.check(self.lib, self._h, self.lib.ibpm_get_forces(self._h, _abi.dptr(s.fb), None))
        self._stale = True


def create_solver(x, **kw) -> AbstractSolver:
    """create_solver(::Problem | ::State; kw...) (solver.jl:28, 152)."""
    state = State(x) if isinstance(x, Problem) else x
    return GpuCnabSolver(state, **kw)


def advance_(solver: AbstractSolver):
    solver.advance_()


def getstate(solver: AbstractSolver) -> State:
    return solver.getstate()


def solve_(solver: AbstractSolver, *, t: float, f: Optional[Callable] = None, save=None, log: bool = False):
    """solve!([f], solver; t, save, log) (solver.jl:37-62)."""
    state = solver.state if hasattr(solver, "state") else solver.getstate()
    n = int(round((t - state.t) / timestep(state.prob)))
    if save is not None:
        save.init(state.index + n)
    try:
        for i in range(1, n + 1):
            solver.advance_()
            if save is not None or f is not None:
                st = solver.getstate()
                if save is not None:
                    save.update(st)
                if f is not None:
                    f(st, i, n)
            if log and i % 10 == 1:
                print("i = ", state.index, "  t = ", state.t)
    finally:
        if save is not None:
            save.finalize()


def solve(prob: Problem, *, t: float, f: Optional[Callable] = None, solver_kw=None, **kw):
    """solve([f], prob; t, save, solver_kw) (solver.jl:71-76)."""
    solver = create_solver(State(prob), **(solver_kw or {}))
    solve_(solver, t=t, f=f, **kw)
    return solver

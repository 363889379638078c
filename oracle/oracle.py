"""ctypes wrapper of the CPU oracle (oracle/ibpm_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker.  The product path never imports it.

`OracleSolver` takes the same `State` objects as the GPU solver
(immersedbodies.jl_b200's host mirror of src/problem.jl) and restates
CnabSolver / advance! (src/solver.jl:84-190) in FP64 on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libibpm_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class orc_problem(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nlevel", C.c_int32),
                ("h", C.c_double), ("x0", C.c_double), ("y0", C.c_double), ("Re", C.c_double), ("dt", C.c_double),
                ("npanel", C.c_int32), ("nbody", C.c_int32), ("body_kind", _ip), ("body_start", _ip),
                ("body_xb", _dp), ("body_ds", _dp), ("grid_moving", C.c_int32),
                ("cg_maxiter", C.c_int32), ("cg_reltol", C.c_double), ("cg_abstol", C.c_double),
                ("timing_only", C.c_int32)]


class orc_step_params(C.Structure):
    _fields_ = [("freestream", C.c_double * 2), ("body_motion", _dp), ("grid_motion", C.c_double * 6)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.POINTER(orc_problem), C.c_char_p, C.c_int]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_advance.restype = C.c_int
    lib.orc_advance.argtypes = [C.c_void_p, C.POINTER(orc_step_params), C.c_char_p, C.c_int]
    for name in ("orc_q", "orc_q0", "orc_gamma", "orc_psi", "orc_xb", "orc_ds", "orc_ub", "orc_fbt", "orc_fb",
                 "orc_freestream"):
        getattr(lib, name).restype = _dp
        getattr(lib, name).argtypes = [C.c_void_p]
    lib.orc_nonlin.restype = _dp
    lib.orc_nonlin.argtypes = [C.c_void_p, C.c_int]
    lib.orc_get_index.restype = C.c_int64
    lib.orc_get_index.argtypes = [C.c_void_p]
    lib.orc_set_index.argtypes = [C.c_void_p, C.c_int64]
    lib.orc_get_t.restype = C.c_double
    lib.orc_get_t.argtypes = [C.c_void_p]
    lib.orc_set_t0.argtypes = [C.c_void_p, C.c_double]
    lib.orc_last_cg_iters.restype = C.c_int
    lib.orc_last_cg_iters.argtypes = [C.c_void_p]
    lib.orc_binv.restype = C.c_int
    lib.orc_binv.argtypes = [C.c_void_p, _dp]
    lib.orc_set_binv.restype = C.c_int
    lib.orc_set_binv.argtypes = [C.c_void_p, _dp]
    lib.orc_apply_B.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_vort2flux.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.orc_reg_rot.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_regT.argtypes = [C.c_void_p, _dp, _dp]
    lib.orc_nthreads.restype = C.c_int
    lib.orc_nthreads.argtypes = [C.c_int]
    lib.orc_dst1.argtypes = [C.c_int, _dp, _dp]
    lib.orc_dst2.argtypes = [C.c_int, C.c_int, _dp, _dp]
    lib.orc_lap_inv.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp]
    lib.orc_lap_eigs.argtypes = [C.c_int, C.c_int, _dp]
    lib.orc_delta_h.restype = C.c_double
    lib.orc_delta_h.argtypes = [C.c_double, C.c_double, C.c_double]
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(_dp)


class OracleError(RuntimeError):
    pass


def dst1(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    load().orc_dst1(len(x), _p(x), _p(y))
    return y


def dst2(x: np.ndarray) -> np.ndarray:
    x = np.asfortranarray(x, dtype=np.float64)
    y = np.empty_like(x, order="F")
    load().orc_dst2(x.shape[0], x.shape[1], _p(x), _p(y))
    return y


def lap_eigs(nx: int, ny: int) -> np.ndarray:
    lam = np.empty((nx - 1, ny - 1), order="F")
    load().orc_lap_eigs(nx, ny, _p(lam))
    return lam


def lap_inv(nx, ny, lam, b):
    lam = np.asfortranarray(lam, dtype=np.float64)
    b = np.asfortranarray(b, dtype=np.float64)
    x = np.empty_like(b, order="F")
    load().orc_lap_inv(nx, ny, _p(lam), _p(b), _p(x))
    return x


def delta_h(rf, rb, dr) -> float:
    return load().orc_delta_h(rf, rb, dr)


def set_threads(n: int) -> int:
    return load().orc_nthreads(n)


class OracleSolver:
    """CnabSolver(state) restated on the CPU; mirrors GpuCnabSolver's methods."""

    def __init__(self, state, *, cg=None, timing_only=False):
        lib = load()
        self.lib = lib
        self.state = state
        prob = state.prob
        bodies = prob.bodies
        kinds = np.array([b.kind for _, b, _ in bodies.preset], dtype=np.int32)
        starts = np.array([r.start for _, _, r in bodies.preset] + [bodies.npanel], dtype=np.int32)
        xb = np.asfortranarray(np.vstack([b.panels.xb for _, b, _ in bodies.preset]))
        ds = np.concatenate([b.panels.ds for _, b, _ in bodies.preset])
        self._keep = (kinds, starts, xb, ds)
        g = prob.grid
        cg = {"maxiter": 5000, "reltol": 1e-12, "abstol": 0.0, **(cg or {})}
        p = orc_problem(nx=g.base.n[0], ny=g.base.n[1], nlevel=g.nlevel, h=g.base.h, x0=g.base.x0[0],
                        y0=g.base.x0[1], Re=prob.fluid.Re, dt=prob.scheme.dt, npanel=bodies.npanel,
                        nbody=len(kinds), body_kind=kinds.ctypes.data_as(_ip), body_start=starts.ctypes.data_as(_ip),
                        body_xb=_p(xb), body_ds=_p(ds), grid_moving=1 if prob.fluid.grid_motion.moving else 0,
                        cg_maxiter=cg["maxiter"], cg_reltol=cg["reltol"], cg_abstol=cg["abstol"],
                        timing_only=1 if timing_only else 0)
        err = C.create_string_buffer(512)
        h = lib.orc_create(C.byref(p), err, 512)
        if not h:
            raise OracleError(err.value.decode())
        self._h = C.c_void_p(h)
        self._moving = [b.kind == 1 for _, b, _ in bodies.preset]
        self._motion = np.zeros((len(kinds), 6))
        # static-body panels were set by _init_body_motion!; copy the rest of the state in
        self._sync_to_oracle(state)

    def __del__(self):
        if getattr(self, "_h", None):
            self.lib.orc_destroy(self._h)
            self._h = None

    def _arr(self, fn, shape, *args):
        ptr = fn(self._h, *args)
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(ptr, shape=(n,)).reshape(shape, order="F")

    def views(self):
        s = self.state
        L = s.prob.grid.nlevel
        nq, ng = s.q.shape[0], s.Gamma.shape[0]
        n = s.prob.bodies.npanel
        lib = self.lib
        return dict(q=self._arr(lib.orc_q, (nq, L)), q0=self._arr(lib.orc_q0, (nq, L)),
                    Gamma=self._arr(lib.orc_gamma, (ng, L)), psi=self._arr(lib.orc_psi, (ng, L)),
                    nonlin0=self._arr(lib.orc_nonlin, (ng, L), 0), nonlin1=self._arr(lib.orc_nonlin, (ng, L), 1),
                    xb=self._arr(lib.orc_xb, (n, 2)), ds=self._arr(lib.orc_ds, (n,)), ub=self._arr(lib.orc_ub, (n, 2)),
                    Fbt=self._arr(lib.orc_fbt, (2 * n,)), fb=self._arr(lib.orc_fb, (2 * n,)),
                    fs=self._arr(lib.orc_freestream, (2,)))

    def _sync_to_oracle(self, s):
        v = self.views()
        v["q"][...] = s.q
        v["q0"][...] = s.q0
        v["Gamma"][...] = s.Gamma
        v["psi"][...] = s.psi
        v["nonlin0"][...] = s.nonlin[0]
        v["nonlin1"][...] = s.nonlin[1]
        for b, (_, body, r) in enumerate(s.prob.bodies.preset):
            if self._moving[b]:
                v["xb"][r.start:r.stop] = s.panels.xb[r.start:r.stop]
                v["ds"][r.start:r.stop] = s.panels.ds[r.start:r.stop]
                v["ub"][r.start:r.stop] = s.panels.ub[r.start:r.stop]
        v["Fbt"][...] = s.Fbt
        v["fs"][...] = s.freestream_vel
        self.lib.orc_set_t0(self._h, s.t0)
        self.lib.orc_set_index(self._h, s.index)
        self.pull()

    def pull(self):
        """Copy the oracle's state into the host State."""
        s = self.state
        v = self.views()
        s.q[...] = v["q"]
        s.q0[...] = v["q0"]
        s.Gamma[...] = v["Gamma"]
        s.psi[...] = v["psi"]
        s.nonlin[0][...] = v["nonlin0"]
        s.nonlin[1][...] = v["nonlin1"]
        s.panels.xb[...] = v["xb"]
        s.panels.ds[...] = v["ds"]
        s.panels.ub[...] = v["ub"]
        s.Fbt[...] = v["Fbt"]
        s.fb[...] = v["fb"].reshape(2, -1).T
        s.freestream_vel = tuple(v["fs"])
        s.index = int(self.lib.orc_get_index(self._h))
        s.t = float(self.lib.orc_get_t(self._h))
        return s

    def advance_(self, pull=True):
        s = self.state
        prob = s.prob
        t = s.t0 + prob.scheme.dt * s.index  # time after inc_time_index!
        prm = orc_step_params()
        fs = prob.fluid.freestream_vel(t)
        prm.freestream[0], prm.freestream[1] = fs
        gm = prob.fluid.grid_motion
        row = gm(t).as_row() if gm.moving else [0.0] * 6
        for k in range(6):
            prm.grid_motion[k] = row[k]
        for b, (_, body, _) in enumerate(prob.bodies.preset):
            if self._moving[b]:
                self._motion[b] = body.motion(t).as_row()
        prm.body_motion = _p(self._motion)
        err = C.create_string_buffer(512)
        if self.lib.orc_advance(self._h, C.byref(prm), err, 512) != 0:
            raise OracleError(err.value.decode())
        if pull:
            self.pull()
        else:
            s.index += 1
            s.t = t

    def getstate(self):
        return self.pull()

    def last_cg_iters(self) -> int:
        return int(self.lib.orc_last_cg_iters(self._h))

    def binv(self):
        n = 2 * self.state.prob.bodies.npanel
        out = np.empty((n, n), order="F")
        return out if self.lib.orc_binv(self._h, _p(out)) else None

    def set_binv(self, m):
        """Replaces the precomputed B^-1 (static bodies) with m (2np x 2np)."""
        m = np.asfortranarray(m, dtype=np.float64)
        if not self.lib.orc_set_binv(self._h, _p(m)):
            raise ValueError("this solver has no precomputed B^-1")

    def apply_B(self, z):
        z = np.ascontiguousarray(z, dtype=np.float64)
        x = np.empty_like(z)
        self.lib.orc_apply_B(self._h, _p(x), _p(z))
        return x

    def vort2flux(self, gamma):
        """vort2flux! on a copy of gamma (ng x L): returns (coarsified gamma, psi, q)."""
        g = np.asfortranarray(gamma, dtype=np.float64).copy(order="F")
        psi = np.zeros_like(g, order="F")
        q = np.zeros((self.state.q.shape[0], g.shape[1]), order="F")
        self.lib.orc_vort2flux(self._h, _p(psi), _p(q), _p(g))
        return g, psi, q

    def reg_rot(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros(self.state.Gamma.shape[0])
        self.lib.orc_reg_rot(self._h, _p(f), _p(out))
        return out

    def regT(self, q1):
        q1 = np.ascontiguousarray(q1, dtype=np.float64)
        out = np.zeros(2 * self.state.prob.bodies.npanel)
        self.lib.orc_regT(self._h, _p(q1), _p(out))
        return out

    def total_force(self):
        return self.state.fb.sum(axis=0)

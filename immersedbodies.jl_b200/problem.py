"""Host-side problem model, mirroring ImmersedBodies.jl's `src/problem.jl`.

These types only describe a problem; no arithmetic of the time step happens
here.  Arrays follow the reference's Julia layouts (column-major, stored as
Fortran-ordered numpy arrays), so `State` buffers can be handed to the C ABI
(`include/ibpm_b200.h`) without reshuffling.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np


def _round_sig1(x: float) -> float:
    """Julia's floor(x; sigdigits=1)."""
    if x == 0:
        return 0.0
    e = math.floor(math.log10(abs(x)))
    m = 10.0 ** e
    return math.floor(x / m) * m


# --- panels and bodies (src/problem.jl:9-261) --------------------------------------------


@dataclasses.dataclass
class Panels:
    """Panel positions `xb` (n x 2) and lengths `ds` (n) (problem.jl:9-12)."""

    xb: np.ndarray
    ds: np.ndarray

    def __post_init__(self):
        self.xb = np.asarray(self.xb, dtype=np.float64).reshape(-1, 2)
        self.ds = np.asarray(self.ds, dtype=np.float64).reshape(-1)
        if self.xb.shape[0] != self.ds.shape[0]:
            raise ValueError("xb and ds have different panel counts")

    @property
    def n(self) -> int:
        return self.xb.shape[0]


@dataclasses.dataclass
class PanelState:
    """Panel positions, lengths and velocities (problem.jl:28-46)."""

    xb: np.ndarray
    ds: np.ndarray
    ub: np.ndarray

    @classmethod
    def zeros(cls, n: int) -> "PanelState":
        return cls(np.zeros((n, 2), order="F"), np.zeros(n), np.zeros((n, 2), order="F"))

    def __eq__(self, other):
        return (np.array_equal(self.xb, other.xb) and np.array_equal(self.ds, other.ds)
                and np.array_equal(self.ub, other.ub))


@dataclasses.dataclass(frozen=True)
class RigidBodyTransform:
    """Position, velocity, angle and angular velocity of a rigid body (problem.jl:241-246)."""

    pos: Tuple[float, float]
    vel: Tuple[float, float]
    angle: float
    angular_vel: float

    def as_row(self) -> List[float]:
        return [self.pos[0], self.pos[1], self.vel[0], self.vel[1], self.angle, self.angular_vel]


class StaticBody:
    """A body fixed in place at `panels` (problem.jl:226-231)."""

    kind = 0

    def __init__(self, panels: Panels):
        self.panels = panels

    @property
    def npanel(self) -> int:
        return self.panels.n


class MovingRigidBody:
    """A non-deforming body whose motion(t) is a RigidBodyTransform (problem.jl:255-261)."""

    kind = 1

    def __init__(self, motion: Callable[[float], RigidBodyTransform], panels: Panels):
        self.motion = motion
        self.panels = panels

    @property
    def npanel(self) -> int:
        return self.panels.n


class Bodies:
    """Named preset bodies, panels stacked in keyword order (problem.jl:136-180)."""

    def __init__(self, bodies: Optional[Dict[str, object]] = None, **kw):
        items = dict(bodies or {})
        items.update(kw)
        if not items:
            raise ValueError("at least one body is required")
        self.byname: Dict[str, Tuple[object, range]] = {}
        self.preset: List[Tuple[str, object, range]] = []
        off = 0
        for name, body in items.items():
            if not isinstance(body, (StaticBody, MovingRigidBody)):
                raise TypeError(f"unsupported body type {type(body).__name__}")
            r = range(off, off + body.npanel)
            off += body.npanel
            self.preset.append((name, body, r))
            self.byname[name] = (body, r)
        self.npanel = off
        self.static = all(isinstance(b, StaticBody) for _, b, _ in self.preset)

    def panel_range(self, name: str) -> range:
        return self.byname[name][1]

    def __getitem__(self, name):
        return self.byname[name][0]


def n_panels(x) -> int:
    if isinstance(x, Bodies):
        return x.npanel
    if isinstance(x, (StaticBody, MovingRigidBody)):
        return x.npanel
    if isinstance(x, (Panels, PanelState)):
        return x.xb.shape[0]
    raise TypeError(type(x))


# --- grids (src/problem.jl:269-475) ------------------------------------------------------


@dataclasses.dataclass(frozen=True)
class CartesianGrid:
    x0: Tuple[float, float]
    n: Tuple[int, int]
    h: float

    @classmethod
    def from_lims(cls, h: float, xlims, ylims) -> "CartesianGrid":
        x0 = (float(xlims[0]), float(ylims[0]))
        n = tuple(int(np.rint((lim[1] - lim[0]) / h)) for lim in (xlims, ylims))
        return cls(x0, n, float(h))


@dataclasses.dataclass(frozen=True)
class GridIndices:
    """Sizes and boundary-array offsets (problem.jl:363-389); offsets are 0-based here."""

    nx: int
    ny: int

    @property
    def nu(self):
        return (self.nx + 1) * self.ny

    @property
    def nv(self):
        return self.nx * (self.ny + 1)

    @property
    def nq(self):
        return self.nu + self.nv

    @property
    def nGamma(self):
        return (self.nx - 1) * (self.ny - 1)

    @property
    def nbc(self):
        return 2 * (self.nx + 1) + 2 * (self.ny + 1)

    L = 0

    @property
    def R(self):
        return self.ny + 1

    @property
    def B(self):
        return 2 * (self.ny + 1)

    @property
    def T(self):
        return 2 * (self.ny + 1) + self.nx + 1


@dataclasses.dataclass(frozen=True)
class MultiDomainGrid:
    base: CartesianGrid
    nlevel: int

    @property
    def inds(self) -> GridIndices:
        return GridIndices(*self.base.n)

    def gridstep(self, level: int = 1) -> float:
        return 2.0 ** (level - 1) * self.base.h

    def subdomain(self, level: int) -> CartesianGrid:
        b = self.base
        h = 2.0 ** (level - 1) * b.h
        x0 = tuple(x + n * (b.h - h) / 2 for x, n in zip(b.x0, b.n))
        return CartesianGrid(x0, b.n, h)


@dataclasses.dataclass(frozen=True)
class MultiDomainExtents:
    xlims: Tuple[float, float]
    ylims: Tuple[float, float]
    nlevel: int


def fluid_grid(*, h=None, xlims, ylims, nlevel):
    """fluid_grid (problem.jl:473-475)."""
    if h is None:
        return MultiDomainExtents(tuple(xlims), tuple(ylims), int(nlevel))
    return MultiDomainGrid(CartesianGrid.from_lims(h, xlims, ylims), int(nlevel))


def default_gridstep(Re: float) -> float:
    return _round_sig1(2.0 / Re)


def coords(grid: CartesianGrid, pts: str = "vertices"):
    """coords(grid, GridU()/GridV()/GridΓ()) (problem.jl:317-344)."""
    xs = grid.x0[0] + grid.h * np.arange(grid.n[0] + 1)
    ys = grid.x0[1] + grid.h * np.arange(grid.n[1] + 1)
    mid = lambda r: r[0] + grid.h / 2 + grid.h * np.arange(len(r) - 1)
    if pts == "vertices":
        return xs, ys
    if pts == "u":
        return xs, mid(ys)
    if pts == "v":
        return mid(xs), ys
    if pts == "gamma":
        return xs[1:-1], ys[1:-1]
    raise ValueError(pts)


# --- fluid, scheme, problem ---------------------------------------------------------------


@dataclasses.dataclass(frozen=True)
class GridVelocity:
    center: Tuple[float, float]
    vel: Tuple[float, float]
    angle: float
    angular_vel: float

    def as_row(self) -> List[float]:
        return [self.center[0], self.center[1], self.vel[0], self.vel[1], self.angle, self.angular_vel]


class StaticGrid:
    moving = False


class MovingGrid:
    moving = True

    def __init__(self, motion: Callable[[float], GridVelocity]):
        self.motion = motion

    def __call__(self, t):
        return self.motion(t)


class Fluid:
    """Fluid(; grid, Re, freestream_vel, grid_motion) (problem.jl:534-552)."""

    def __init__(self, *, grid, Re, freestream_vel=lambda t: (0.0, 0.0), grid_motion=None):
        if isinstance(grid, MultiDomainExtents):
            grid = fluid_grid(h=default_gridstep(Re), xlims=grid.xlims, ylims=grid.ylims, nlevel=grid.nlevel)
        self.grid: MultiDomainGrid = grid
        self.Re = float(Re)
        self.freestream_vel = freestream_vel
        self.grid_motion = grid_motion if grid_motion is not None else StaticGrid()


class CNAB:
    """2-step Crank-Nicolson/Adams-Bashforth scheme (problem.jl:566-577)."""

    def __init__(self, *, dt, n=2):
        if n != 2:
            raise ValueError("only 2-step CNAB is currently supported")
        self.dt = float(dt)
        self.beta = (1.5, -0.5)


def default_scheme(grid, *, Umax, cfl=0.1) -> CNAB:
    """default_scheme (problem.jl:590-596)."""
    h = grid.gridstep() if isinstance(grid, MultiDomainGrid) else grid.h
    return CNAB(dt=_round_sig1(cfl * h / Umax))


def timestep(x) -> float:
    if isinstance(x, Problem):
        return x.scheme.dt
    return x.dt


class Problem:
    def __init__(self, *, fluid: Fluid, bodies: Bodies, scheme: CNAB):
        self.fluid = fluid
        self.bodies = bodies
        self.scheme = scheme

    @property
    def grid(self) -> MultiDomainGrid:
        return self.fluid.grid


# --- state (src/problem.jl:626-708) -------------------------------------------------------


class State:
    """State(prob; t0=0) (problem.jl:626-665); arrays are Fortran-ordered."""

    def __init__(self, prob: Problem, t0: float = 0.0):
        inds = prob.grid.inds
        L = prob.grid.nlevel
        n = prob.bodies.npanel
        self.prob = prob
        self.t0 = float(t0)
        self.q = np.zeros((inds.nq, L), order="F")
        self.q0 = np.zeros((inds.nq, L), order="F")
        self.Gamma = np.zeros((inds.nGamma, L), order="F")
        self.psi = np.zeros((inds.nGamma, L), order="F")
        self.nonlin = [np.zeros((inds.nGamma, L), order="F") for _ in prob.scheme.beta]
        self.panels = PanelState.zeros(n)
        self.Fbt = np.zeros(2 * n)
        self.fb = np.zeros((n, 2), order="F")
        self.freestream_vel = (0.0, 0.0)
        set_time_index_(self, 0)

    def __eq__(self, o):
        return (self.prob is o.prob and self.index == o.index and self.t == o.t and self.t0 == o.t0
                and all(np.array_equal(getattr(self, k), getattr(o, k)) for k in ("q", "q0", "Gamma", "psi", "Fbt", "fb"))
                and all(np.array_equal(a, b) for a, b in zip(self.nonlin, o.nonlin))
                and self.panels == o.panels and tuple(self.freestream_vel) == tuple(o.freestream_vel))


def set_time_index_(state: State, index: int):
    """set_time_index! (problem.jl:705-708): t = t0 + dt (index - 1)."""
    state.index = int(index)
    state.t = state.t0 + timestep(state.prob) * (index - 1)


def inc_time_index_(state: State):
    set_time_index_(state, state.index + 1)


def update_vars_(state: State):
    """update_vars! (problem.jl:676-685): fb = F~b h / dt."""
    prob = state.prob
    state.fb[:] = state.Fbt.reshape(2, -1).T * prob.grid.gridstep() / timestep(prob)


# --- accessors (src/problem.jl:715-866) ---------------------------------------------------


def _split_flux(q, inds: GridIndices):
    u = q[: inds.nu].reshape((inds.nx + 1, inds.ny) + q.shape[1:], order="F")
    v = q[inds.nu:].reshape((inds.nx, inds.ny + 1) + q.shape[1:], order="F")
    return u, v


def x_velocity(state: State) -> np.ndarray:
    g = state.prob.grid
    u, _ = _split_flux(state.q + state.q0, g.inds)
    return np.stack([u[..., l] / g.gridstep(l + 1) for l in range(g.nlevel)], axis=-1)


def y_velocity(state: State) -> np.ndarray:
    g = state.prob.grid
    _, v = _split_flux(state.q + state.q0, g.inds)
    return np.stack([v[..., l] / g.gridstep(l + 1) for l in range(g.nlevel)], axis=-1)


def vorticity(state: State) -> np.ndarray:
    g = state.prob.grid
    i = g.inds
    G = state.Gamma.reshape((i.nx - 1, i.ny - 1, g.nlevel), order="F")
    return np.stack([G[..., l] / g.gridstep(l + 1) ** 2 for l in range(g.nlevel)], axis=-1)


def boundary_force(state: State, body: Optional[str] = None) -> np.ndarray:
    if body is None:
        return state.fb
    return state.fb[list(state.prob.bodies.panel_range(body)), :]


def boundary_total_force(state: State, body: Optional[str] = None) -> np.ndarray:
    return boundary_force(state, body).sum(axis=0)

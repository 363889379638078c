"""The benchmark and parity workloads, built with the host API.

Each builder returns a `Problem` plus any initial-state setup.  Inputs are
synthetic and seeded (no dataset is involved):
  cylinder_re100_200      200 x 200, 3 levels, 157 points, Re 100, dt 0.004 (the CPU-runnable case)
  cylinder_re100_1024     1024 x 1024, 5 levels, 628 points, Re 100, dt 0.001, Γ noise 1e-3 (seed 12345)
  plate_aoa30_1024        1024 x 1024, 5 levels, 201-point flat plate at 30 deg, Re 200, dt 0.001
  pitching_plate_512      512 x 512, 4 levels, 101-point plate pitching/plunging, Re 500, dt 0.002
  ensemble_cases          seeded cases of {256, 384, 512} x 256 cells, 3 levels, cylinders or plates (seed 2026)
  small_cylinder          a few-second case for tests (any size)
"""
from __future__ import annotations

import math

import numpy as np

from . import curves as Curves
from .problem import (CNAB, Bodies, Fluid, MovingRigidBody, Problem, RigidBodyTransform, State, StaticBody,
                      fluid_grid)


def uniform_flow(t):
    return (1.0, 0.0)


def cylinder(h, xlims, ylims, nlevel, npts, Re, dt, r=0.5, center=(0.0, 0.0)) -> Problem:
    fluid = Fluid(grid=fluid_grid(h=h, xlims=xlims, ylims=ylims, nlevel=nlevel), Re=Re, freestream_vel=uniform_flow)
    panels = Curves.partition(Curves.Circle(r=r, center=center), int(npts))
    return Problem(fluid=fluid, bodies=Bodies(cyl=StaticBody(panels)), scheme=CNAB(dt=dt))


def cylinder_re100_200() -> Problem:
    return cylinder(0.02, (-1.0, 3.0), (-2.0, 2.0), 3, 157, 100.0, 0.004)


def cylinder_re100_1024() -> Problem:
    return cylinder(0.005, (-1.56, 3.56), (-2.56, 2.56), 5, 628, 100.0, 0.001)


def seed_vorticity(state: State, amplitude: float = 1e-3, seed: int = 12345):
    """Γ = N(0,1) * amplitude * hc^2 on every level (vorticity noise of the given amplitude)."""
    g = state.prob.grid
    rng = np.random.default_rng(seed)
    for lev in range(g.nlevel):
        hc = g.gridstep(lev + 1)
        state.Gamma[:, lev] = rng.standard_normal(state.Gamma.shape[0]) * amplitude * hc * hc
    return state


def plate(h, xlims, ylims, nlevel, npts, Re, dt, aoa_deg, chord=1.0) -> Problem:
    fluid = Fluid(grid=fluid_grid(h=h, xlims=xlims, ylims=ylims, nlevel=nlevel), Re=Re, freestream_vel=uniform_flow)
    a = math.radians(aoa_deg)
    c, s = 0.5 * chord * math.cos(a), 0.5 * chord * math.sin(a)
    panels = Curves.partition(Curves.LineSegment((-c, s), (c, -s)), int(npts))
    return Problem(fluid=fluid, bodies=Bodies(plate=StaticBody(panels)), scheme=CNAB(dt=dt))


def plate_aoa30_1024() -> Problem:
    return plate(0.005, (-1.56, 3.56), (-2.56, 2.56), 5, 201, 200.0, 0.001, 30.0)


def pitching_plate(k: float = 0.5, h=0.01, n=512, nlevel=4, npts=101, Re=500.0, dt=0.002,
                   theta0_deg=30.0, plunge=0.25) -> Problem:
    """Plate of chord 1 pitching about mid-chord θ(t) = θ0 sin(2πft) and plunging
    y(t) = plunge sin(2πft), with reduced frequency k = π f / U (U = 1)."""
    span = n * h
    fluid = Fluid(grid=fluid_grid(h=h, xlims=(-0.3 * span, 0.7 * span), ylims=(-0.5 * span, 0.5 * span),
                                  nlevel=nlevel), Re=Re, freestream_vel=uniform_flow)
    f = k / math.pi
    th0 = math.radians(theta0_deg)
    w = 2 * math.pi * f

    def motion(t):
        return RigidBodyTransform(pos=(0.0, plunge * math.sin(w * t)), vel=(0.0, plunge * w * math.cos(w * t)),
                                  angle=-th0 * math.sin(w * t), angular_vel=-th0 * w * math.cos(w * t))

    panels = Curves.partition(Curves.LineSegment((-0.5, 0.0), (0.5, 0.0)), int(npts))
    return Problem(fluid=fluid, bodies=Bodies(plate=MovingRigidBody(motion, panels)), scheme=CNAB(dt=dt))


def small_cylinder(n=64, nlevel=3, npts=None, Re=100.0, dt=None) -> Problem:
    """A scaled-down config-1 cylinder for fast parity tests."""
    h = 4.0 / n
    npts = npts or max(16, int(round(math.pi / h)))
    return cylinder(h, (-1.0, 3.0), (-2.0, 2.0), nlevel, npts, Re, dt or 0.2 * h)


def ensemble_cases(n: int = 128, seed: int = 2026, h: float = 0.01, nlevel: int = 3, dt: float = 0.002,
                   widths=(256, 384, 512), ny: int = 256):
    """n independent cases from a seeded generator: a finest grid of nx x ny
    cells (nx drawn from `widths`) at spacing h with `nlevel` levels; a static
    cylinder of diameter D ~ U[0.5, 1.5] or a flat plate of chord 1 at an angle
    of attack ~ U[0, 45] deg, with body points about h apart; Re ~ U[50, 300];
    uniform flow (1, 0).  Returns the list of Problems."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.choice(widths))
        Re = float(rng.uniform(50.0, 300.0))
        W, H = nx * h, ny * h
        xlims, ylims = (-0.4 * H, -0.4 * H + W), (-0.5 * H, 0.5 * H)
        fluid = Fluid(grid=fluid_grid(h=h, xlims=xlims, ylims=ylims, nlevel=nlevel), Re=Re,
                      freestream_vel=uniform_flow)
        if rng.uniform() < 0.5:
            D = float(rng.uniform(0.5, 1.5))
            panels = Curves.partition(Curves.Circle(r=D / 2, center=(0.0, 0.0)), int(round(math.pi * D / h)))
            body = Bodies(cyl=StaticBody(panels))
        else:
            aoa = math.radians(float(rng.uniform(0.0, 45.0)))
            c, s = 0.5 * math.cos(aoa), 0.5 * math.sin(aoa)
            panels = Curves.partition(Curves.LineSegment((-c, s), (c, -s)), int(round(1.0 / h)))
            body = Bodies(plate=StaticBody(panels))
        out.append(Problem(fluid=fluid, bodies=body, scheme=CNAB(dt=dt)))
    return out

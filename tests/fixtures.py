"""Rebuilds the golden-fixture problems (tests/golden/make_golden.py) with the host API."""
from __future__ import annotations

import math

import numpy as np


def problem_from_fixture(ib, fx):
    nx, L = int(fx["nx"]), int(fx["L"])
    h = 4.0 / nx
    kind = str(fx["kind"])
    grid_moving = bool(int(fx["grid_moving"]))
    gm = None
    if grid_moving:
        gm = ib.MovingGrid(lambda t: ib.GridVelocity(center=(-1.0, 0.0), vel=(0.0, 0.2), angle=0.1 * math.sin(t),
                                                     angular_vel=0.1 * math.cos(t)))
    fluid = ib.Fluid(grid=ib.fluid_grid(h=h, xlims=(-1.0, 3.0), ylims=(-2.0, 2.0), nlevel=L), Re=float(fx["Re"]),
                     freestream_vel=lambda t: (1.0, 0.0), grid_motion=gm)
    xb = np.asarray(fx["xb"])
    panels = ib.Panels(xb, np.full(xb.shape[0], 0.1))
    if kind == "moving":
        w = 2.0

        def motion(t):
            return ib.RigidBodyTransform(pos=(0.0, 0.1 * math.sin(w * t)), vel=(0.0, 0.1 * w * math.cos(w * t)),
                                         angle=-0.2 * math.sin(w * t), angular_vel=-0.2 * w * math.cos(w * t))

        body = ib.MovingRigidBody(motion, panels)
    else:
        body = ib.StaticBody(panels)
    prob = ib.Problem(fluid=fluid, bodies=ib.Bodies(body=body), scheme=ib.CNAB(dt=float(fx["dt"])))
    state = ib.State(prob)
    state.Gamma[...] = fx["Gamma0"]
    return prob, state


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d

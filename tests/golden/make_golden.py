"""Independent numpy/scipy transcription of ImmersedBodies.jl's advance! and the
golden-fixture generator for the parity tests.

The reference (Julia) cannot run in this container, so this file restates
src/fluid.jl, src/coupling.jl, src/bodies.jl and src/solver.jl a second time,
vectorised with numpy, with scipy.fft.dstn(type=1) as the 2D DST-I (the same
unnormalised definition as FFTW's RODFT00 used at src/fluid.jl:113-115) and
numpy.linalg.inv for inv(B).  It shares no code with the C oracle
(oracle/ibpm_oracle.c); the tests check the two against each other and keep
the fixtures this script writes.

Run:  python tests/golden/make_golden.py        (writes tests/golden/*.npz)
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np
import scipy.fft as sf

HERE = os.path.dirname(os.path.abspath(__file__))


class Grid:
    def __init__(self, nx, ny, L, h, x0, y0):
        self.nx, self.ny, self.L, self.h, self.x0, self.y0 = nx, ny, L, h, x0, y0
        self.nu = (nx + 1) * ny
        self.nq = self.nu + nx * (ny + 1)
        self.ng = (nx - 1) * (ny - 1)

    def hc(self, lev):
        return 2.0 ** (lev - 1) * self.h

    def split(self, q):
        return (q[: self.nu].reshape(self.nx + 1, self.ny, order="F"),
                q[self.nu:].reshape(self.nx, self.ny + 1, order="F"))

    def G2(self, g):
        return g.reshape(self.nx - 1, self.ny - 1, order="F")


def flat(a):
    return a.reshape(-1, order="F")


# --- fluid.jl -----------------------------------------------------------------------------

def rot(gr, q):  # fluid.jl:101-111
    qx, qy = gr.split(q)
    return flat((qx[1:gr.nx, 0:gr.ny - 1] - qx[1:gr.nx, 1:gr.ny]) + (qy[1:gr.nx, 1:gr.ny] - qy[0:gr.nx - 1, 1:gr.ny]))


def get_bc(gr, r):  # fluid.jl:278-306 -> dict of side arrays indexed by ibc (1-based; index 0 unused)
    nx, ny = gr.nx, gr.ny
    R = gr.G2(r)
    B = np.zeros(nx + 2)
    T = np.zeros(nx + 2)
    Lf = np.zeros(ny + 2)
    Rt = np.zeros(ny + 2)
    k = np.arange(0, nx // 2 + 1)
    i = nx // 4 + k
    B[1 + 2 * k] = R[i - 1, ny // 4 - 1]
    T[1 + 2 * k] = R[i - 1, 3 * ny // 4 - 1]
    k = np.arange(1, nx // 2 + 1)
    i = nx // 4 + k
    B[2 * k] = 0.5 * (R[i - 1, ny // 4 - 1] + R[i - 2, ny // 4 - 1])
    T[2 * k] = 0.5 * (R[i - 1, 3 * ny // 4 - 1] + R[i - 2, 3 * ny // 4 - 1])
    k = np.arange(0, ny // 2 + 1)
    j = ny // 4 + k
    Lf[1 + 2 * k] = R[nx // 4 - 1, j - 1]
    Rt[1 + 2 * k] = R[3 * nx // 4 - 1, j - 1]
    k = np.arange(1, ny // 2 + 1)
    j = ny // 4 + k
    Lf[2 * k] = 0.5 * (R[nx // 4 - 1, j - 1] + R[nx // 4 - 1, j - 2])
    Rt[2 * k] = 0.5 * (R[3 * nx // 4 - 1, j - 1] + R[3 * nx // 4 - 1, j - 2])
    return dict(B=B, T=T, L=Lf, R=Rt)


def zero_bc(gr):
    return dict(B=np.zeros(gr.nx + 2), T=np.zeros(gr.nx + 2), L=np.zeros(gr.ny + 2), R=np.zeros(gr.ny + 2))


def scale_bc(bc, f):
    return {k: v * f for k, v in bc.items()}


def apply_bc(gr, r, bc, fac):  # fluid.jl:308-338
    R = gr.G2(r.copy())
    nx, ny = gr.nx, gr.ny
    i = np.arange(1, nx)
    R[i - 1, 0] += fac * bc["B"][i + 1]
    R[i - 1, ny - 2] += fac * bc["T"][i + 1]
    j = np.arange(1, ny)
    R[0, j - 1] += fac * bc["L"][j + 1]
    R[nx - 2, j - 1] += fac * bc["R"][j + 1]
    return flat(R)


def curl(gr, psi, bc):  # fluid.jl:230-276
    nx, ny = gr.nx, gr.ny
    P = gr.G2(psi)
    qx = np.zeros((nx + 1, ny))
    qy = np.zeros((nx, ny + 1))
    qx[1:nx, 1:ny - 1] = P[0:nx - 1, 1:ny - 1] - P[0:nx - 1, 0:ny - 2]
    i = np.arange(2, nx + 1)
    qx[i - 1, 0] = P[i - 2, 0] - bc["B"][i]
    qx[i - 1, ny - 1] = bc["T"][i] - P[i - 2, ny - 2]
    j = np.arange(1, ny + 1)
    qx[0, j - 1] = bc["L"][j + 1] - bc["L"][j]
    qx[nx, j - 1] = bc["R"][j + 1] - bc["R"][j]
    qy[1:nx - 1, 1:ny] = P[0:nx - 2, 0:ny - 1] - P[1:nx - 1, 0:ny - 1]
    j = np.arange(2, ny + 1)
    qy[0, j - 1] = bc["L"][j] - P[0, j - 2]
    qy[nx - 1, j - 1] = P[nx - 2, j - 2] - bc["R"][j]
    i = np.arange(1, nx + 1)
    qy[i - 1, 0] = bc["B"][i] - bc["B"][i + 1]
    qy[i - 1, ny] = bc["T"][i] - bc["T"][i + 1]
    return np.concatenate([flat(qx), flat(qy)])


def coarsify(gr, Gc, G):  # fluid.jl:208-228
    nx, ny = gr.nx, gr.ny
    F = gr.G2(G)
    C = gr.G2(Gc.copy())
    is_ = nx // 2 + np.arange(-nx // 2 + 2, nx // 2 - 2 + 1, 2)
    js = ny // 2 + np.arange(-ny // 2 + 2, ny // 2 - 2 + 1, 2)
    ics = nx // 2 + np.arange(-nx // 4 + 1, nx // 4 - 1 + 1)
    jcs = ny // 2 + np.arange(-ny // 4 + 1, ny // 4 - 1 + 1)
    n_i, n_j = min(len(is_), len(ics)), min(len(js), len(jcs))
    I, J = np.meshgrid(is_[:n_i] - 1, js[:n_j] - 1, indexing="ij")
    IC, JC = np.meshgrid(ics[:n_i] - 1, jcs[:n_j] - 1, indexing="ij")
    C[IC, JC] = (F[I, J] + 0.5 * (F[I + 1, J] + F[I, J + 1] + F[I - 1, J] + F[I, J - 1])
                 + 0.25 * (F[I + 1, J + 1] + F[I + 1, J - 1] + F[I - 1, J - 1] + F[I - 1, J + 1]))
    return flat(C)


def lap_eigs(gr):  # fluid.jl:168-173
    i = np.arange(1, gr.nx)[:, None]
    j = np.arange(1, gr.ny)[None, :]
    return -2 * (np.cos(np.pi * i / gr.nx) + np.cos(np.pi * j / gr.ny) - 2)


def lap_inv(gr, Lam, b):  # fluid.jl:145-166
    scale = 1 / (4 * gr.nx * gr.ny)
    t = sf.dstn(gr.G2(b), type=1)
    t = t * (scale / Lam)
    return flat(sf.dstn(t, type=1))


def vort2flux(gr, lam, G, curl_levels=True):  # fluid.jl:178-205; G (ng x L) modified in place
    L = gr.L
    for lev in range(2, L + 1):
        G[:, lev - 1] = coarsify(gr, G[:, lev - 1], G[:, lev - 2])
    psi = np.zeros_like(G)
    q = np.zeros((gr.nq, L))
    psi[:, L - 1] = lap_inv(gr, lam, G[:, L - 1])
    q[:, L - 1] = curl(gr, psi[:, L - 1], zero_bc(gr))
    for lev in range(L - 1, 0, -1):
        bc = get_bc(gr, psi[:, lev])
        tmp = apply_bc(gr, G[:, lev - 1], bc, 1.0)
        psi[:, lev - 1] = lap_inv(gr, lam, tmp)
        q[:, lev - 1] = curl(gr, psi[:, lev - 1], bc)
    return psi, q


def base_flux(gr, fs, lev, gm=None):  # fluid.jl:22-67
    hc = gr.hc(lev)
    if gm is None:
        return np.concatenate([np.full(gr.nu, fs[0] * hc), np.full(gr.nq - gr.nu, fs[1] * hc)])
    cx, cy, u0x, u0y, th, Om = gm
    ct, st = math.cos(th), math.sin(th)
    x0 = gr.x0 + gr.nx * (gr.h - hc) / 2
    y0 = gr.y0 + gr.ny * (gr.h - hc) / 2

    def w(x, y):
        dx, dy = x - cx, y - cy
        wx = fs[0] - u0x - ((Om * -st) * dx + (Om * -ct) * dy)
        wy = fs[1] - u0y - ((Om * ct) * dx + (Om * -st) * dy)
        return wx, wy

    xu = x0 + hc * np.arange(gr.nx + 1)
    yu = y0 + hc / 2 + hc * np.arange(gr.ny)
    X, Y = np.meshgrid(xu, yu, indexing="ij")
    wx, wy = w(X, Y)
    qx = hc * (ct * wx + st * wy)
    xv = x0 + hc / 2 + hc * np.arange(gr.nx)
    yv = y0 + hc * np.arange(gr.ny + 1)
    X, Y = np.meshgrid(xv, yv, indexing="ij")
    wx, wy = w(X, Y)
    qy = hc * (-st * wx + ct * wy)
    return np.concatenate([flat(qx), flat(qy)])


def nonlinear(gr, q, q0, G, bc, lev):  # fluid.jl:340-455
    nx, ny = gr.nx, gr.ny
    qx, qy = gr.split(q)
    q0x, q0y = gr.split(q0)
    Qx = np.zeros((nx + 1, ny))
    Qy = np.zeros((nx, ny + 1))
    Qx[:, 1:] = (qx[:, 1:] + qx[:, :-1] + q0x[:, 1:] + q0x[:, :-1]) / 2
    Qy[1:, :] = (qy[1:, :] + qy[:-1, :] + q0y[1:, :] + q0y[:-1, :]) / 2
    Gm = gr.G2(G)
    fqx = np.zeros((nx + 1, ny))
    fqy = np.zeros((nx, ny + 1))
    fqx[1:nx, 1:ny - 1] = (Qy[1:nx, 2:ny] * Gm[0:nx - 1, 1:ny - 1] + Qy[1:nx, 1:ny - 1] * Gm[0:nx - 1, 0:ny - 2]) / 2
    i = np.arange(2, nx + 1)
    fqx[i - 1, 0] = (Qy[i - 1, 1] * Gm[i - 2, 0] + Qy[i - 1, 0] * bc["B"][i]) / 2
    fqx[i - 1, ny - 1] = (Qy[i - 1, ny - 1] * Gm[i - 2, ny - 2] + Qy[i - 1, ny] * bc["T"][i]) / 2
    fqy[1:nx - 1, 1:ny] = -(Qx[2:nx, 1:ny] * Gm[1:nx - 1, 0:ny - 1] + Qx[1:nx - 1, 1:ny] * Gm[0:nx - 2, 0:ny - 1]) / 2
    j = np.arange(2, ny + 1)
    fqy[0, j - 1] = -(Qx[1, j - 1] * Gm[0, j - 2] + Qx[0, j - 1] * bc["L"][j]) / 2
    fqy[nx - 1, j - 1] = -(Qx[nx - 1, j - 1] * Gm[nx - 2, j - 2] + Qx[nx, j - 1] * bc["R"][j]) / 2
    hc = gr.hc(lev)
    return rot(gr, np.concatenate([flat(fqx), flat(fqy)])) * (1 / hc ** 2)


# --- coupling.jl --------------------------------------------------------------------------

def delta_h(rf, rb, dr):  # coupling.jl:91-148 (Yang et al., JCP 2009), vectorised
    r1 = np.abs(np.asarray(rf, dtype=float) - rb) / dr
    r2, r3, r4 = r1 ** 2, r1 ** 3, r1 ** 4
    out = np.zeros_like(r1)
    with np.errstate(invalid="ignore"):
        a5 = np.arcsin(0.5 * np.sqrt(3.0) * (2.0 * r1 - 1.0))
        a8 = np.sqrt(1.0 - 12.0 * r2 + 12.0 * r1)
        v1 = (4.166666667e-2 * r4 + (-0.1388888889 + 3.472222222e-2 * a8) * r3
              + (-7.121664902e-2 - 5.208333333e-2 * a8 + 0.2405626122 * a5) * r2
              + (-0.2405626122 * a5 - 0.3792313933 + 0.1012731481 * a8) * r1
              + 8.0187537413e-2 * a5 - 4.195601852e-2 * a8 + 0.6485698427)
        a6 = np.arcsin(0.5 * np.sqrt(3.0) * (-3.0 + 2.0 * r1))
        a9 = np.sqrt(-23.0 + 36.0 * r1 - 12.0 * r2)
        v2 = (-6.25e-2 * r4 + (0.4861111111 - 1.736111111e-2 * a9) * r3
              + (-1.143175026 + 7.8125e-2 * a9 - 0.1202813061 * a6) * r2
              + (0.8751991178 + 0.3608439183 * a6 - 0.1548032407 * a9) * r1 - 0.2806563809 * a6
              + 8.22848104e-3 + 0.1150173611 * a9)
        a1 = np.arcsin(0.5 * (2.0 * r1 - 5.0) * np.sqrt(3.0))
        a7 = np.sqrt(-71.0 - 12.0 * r2 + 60.0 * r1)
        v3 = (2.083333333e-2 * r4 + (3.472222222e-3 * a7 - 0.2638888889) * r3
              + (1.214391675 - 2.604166667e-2 * a7 + 2.405626122e-2 * a1) * r2
              + (-0.1202813061 * a1 - 2.449273192 + 7.262731481e-2 * a7) * r1 + 0.1523563211 * a1
              + 1.843201677 - 7.306134259e-2 * a7)
    out = np.where(r1 <= 1.0, v1, np.where(r1 <= 2.0, v2, np.where(r1 <= 3.0, v3, 0.0)))
    return out


class Reg:  # coupling.jl:3-54
    def __init__(self, gr, np_):
        self.gr = gr
        self.pc = np.zeros((np_, 2), dtype=int)
        self.w = np.zeros((np_, 2, 7, 7))

    def update(self, idx, xb, yb):
        gr = self.gr
        ix = int(np.rint((xb - gr.x0) / gr.h + 1.0 - 0.25))
        iy = int(np.rint((yb - gr.y0) / gr.h + 1.0 - 0.25))
        for i, n in ((ix, gr.nx), (iy, gr.ny)):
            if not (3 < i <= n - 3):
                raise ValueError(f"Panel index={idx + 1} at ({xb}, {yb}) outside allowed region")
        self.pc[idx] = (ix, iy)
        k = np.arange(-3, 4)
        x = gr.x0 + gr.h * ((ix + k) - 1)
        y = gr.y0 + gr.h * ((iy + k) - 1)
        self.w[idx, 0] = delta_h(x, xb, gr.h)[:, None] * delta_h(y + gr.h / 2, yb, gr.h)[None, :]
        self.w[idx, 1] = delta_h(x + gr.h / 2, xb, gr.h)[:, None] * delta_h(y, yb, gr.h)[None, :]

    def regT(self, q):  # coupling.jl:57-69
        qx, qy = self.gr.split(q)
        n = len(self.pc)
        f = np.zeros(2 * n)
        for p, (ix, iy) in enumerate(self.pc):
            f[p] = np.sum(qx[ix - 4:ix + 3, iy - 4:iy + 3] * self.w[p, 0])
            f[n + p] = np.sum(qy[ix - 4:ix + 3, iy - 4:iy + 3] * self.w[p, 1])
        return f

    def reg(self, f):  # coupling.jl:72-85
        gr = self.gr
        qx = np.zeros((gr.nx + 1, gr.ny))
        qy = np.zeros((gr.nx, gr.ny + 1))
        n = len(self.pc)
        for p, (ix, iy) in enumerate(self.pc):
            qx[ix - 4:ix + 3, iy - 4:iy + 3] += self.w[p, 0] * f[p]
            qy[ix - 4:ix + 3, iy - 4:iy + 3] += self.w[p, 1] * f[n + p]
        return np.concatenate([flat(qx), flat(qy)])


# --- solver.jl ----------------------------------------------------------------------------

class Solver:
    """CnabSolver + advance! (solver.jl:84-190) for static bodies (precomputed inv(B)),
    moving rigid bodies (CG) and either grid motion."""

    def __init__(self, nx, ny, L, h, x0, y0, Re, dt, xb_ref, body_slices, body_moving, grid_moving=False,
                 cg_maxiter=5000, cg_reltol=1e-12):
        self.gr = gr = Grid(nx, ny, L, h, x0, y0)
        self.Re, self.dt = Re, dt
        self.np = n = xb_ref.shape[0]
        self.xb_ref = xb_ref
        self.slices, self.moving = body_slices, body_moving
        self.grid_moving = grid_moving
        self.cg_maxiter, self.cg_reltol = cg_maxiter, cg_reltol
        self.lam = lap_eigs(gr)
        self.Lexpl, self.Limpl = [], []
        for lev in range(1, L + 1):
            hc = gr.hc(lev)
            self.Lexpl.append(1.0 / (1 - self.lam * dt / (2 * Re * hc ** 2)))
            self.Limpl.append(1 + self.lam * dt / (2 * Re * hc ** 2))
        self.reg = Reg(gr, n)
        self.xb = np.zeros((n, 2))
        self.ub = np.zeros((n, 2))
        for sl, mv in zip(body_slices, body_moving):
            if not mv:
                self.xb[sl] = xb_ref[sl]
                for p in range(sl.start, sl.stop):
                    self.reg.update(p, *self.xb[p])
        self.index, self.t0 = 0, 0.0
        self.q = np.zeros((gr.nq, L))
        self.q0 = np.zeros((gr.nq, L))
        self.G = np.zeros((gr.ng, L))
        self.psi = np.zeros((gr.ng, L))
        self.nonlin = [np.zeros((gr.ng, L)), np.zeros((gr.ng, L))]
        self.Fbt = np.zeros(2 * n)
        self.Binv = None
        if not any(body_moving):
            Bm = np.column_stack([self.B(np.eye(2 * n)[:, i]) for i in range(2 * n)])
            self.Binv = np.linalg.inv(Bm)

    def B(self, z):  # coupling.jl:163-176
        gr = self.gr
        Gt = np.zeros((gr.ng, gr.L))
        Gt[:, 0] = lap_inv(gr, self.Limpl[0], rot(gr, self.reg.reg(z)))
        _, q = vort2flux(gr, self.lam, Gt)
        return self.reg.regT(q[:, 0])

    def cg(self, x, b):  # IterativeSolvers.jl cg! as called at coupling.jl:198-201
        r = b - self.B(x)
        res = np.linalg.norm(r)
        tol = self.cg_reltol * res
        u = np.zeros_like(x)
        prev = 1.0
        it = 0
        while not (it >= self.cg_maxiter or res <= tol):
            u = r + (res ** 2 / prev ** 2) * u
            c = self.B(u)
            alpha = res ** 2 / np.dot(u, c)
            x = x + alpha * u
            r = r - alpha * c
            prev, res = res, np.linalg.norm(r)
            it += 1
        return x, it

    def advance(self, fs, body_motion=None, grid_motion=None):  # solver.jl:155-190
        gr, dt, Re, L = self.gr, self.dt, self.Re, self.gr.L
        self.index += 1
        for b, (sl, mv) in enumerate(zip(self.slices, self.moving)):  # bodies.jl:12-31
            if mv:
                r0x, r0y, v0x, v0y, ang, Om = body_motion[b]
                c, s = math.cos(ang), math.sin(ang)
                rx, ry = self.xb_ref[sl, 0], self.xb_ref[sl, 1]
                self.xb[sl, 0] = r0x + (c * rx + -s * ry)
                self.xb[sl, 1] = r0y + (s * rx + c * ry)
                self.ub[sl, 0] = v0x + ((Om * -s) * rx + (Om * -c) * ry)
                self.ub[sl, 1] = v0y + ((Om * c) * rx + (Om * -s) * ry)
                for p in range(sl.start, sl.stop):
                    self.reg.update(p, *self.xb[p])
        for lev in range(1, L + 1):
            self.q0[:, lev - 1] = base_flux(gr, fs, lev, grid_motion if self.grid_moving else None)
        # get_trial_state (fluid.jl:467-506)
        Gs = np.zeros_like(self.G)
        for lev in range(L, 0, -1):
            hc = gr.hc(lev)
            rhsbc = np.zeros(gr.ng)
            bc = zero_bc(gr)
            if lev < L:
                bc = get_bc(gr, self.G[:, lev])
                rhsbc = apply_bc(gr, rhsbc, bc, 0.25 * dt / (Re * hc ** 2))
            bc = scale_bc(bc, 0.25)
            self.nonlin[0][:, lev - 1] = nonlinear(gr, self.q[:, lev - 1], self.q0[:, lev - 1], self.G[:, lev - 1],
                                                   bc, lev)
            rhs = lap_inv(gr, self.Lexpl[lev - 1], self.G[:, lev - 1])
            rhs = rhs + dt * 1.5 * self.nonlin[0][:, lev - 1]
            rhs = rhs + dt * -0.5 * self.nonlin[1][:, lev - 1]
            rhs = rhs + rhsbc
            Gs[:, lev - 1] = lap_inv(gr, self.Limpl[lev - 1], rhs)
        self.nonlin = [self.nonlin[1], self.nonlin[0]]
        self.psi, qs = vort2flux(gr, self.lam, Gs)
        # couple_surface_rigid (coupling.jl:236-250)
        F = self.reg.regT(qs[:, 0] + self.q0[:, 0]) - flat(self.ub) * gr.h
        if self.Binv is not None:
            self.Fbt = self.Binv @ F
            self.cg_iters = 0
        else:
            self.Fbt, self.cg_iters = self.cg(self.Fbt.copy(), F)
        # project_circ (coupling.jl:218-230)
        self.G = Gs.copy()
        self.G[:, 0] -= lap_inv(gr, self.Limpl[0], rot(gr, self.reg.reg(self.Fbt)))
        self.psi, self.q = vort2flux(gr, self.lam, self.G)
        self.fb = self.Fbt.reshape(2, -1).T * gr.h / dt


def make_case(name, nx, L, npts, Re, dt, nsteps, kind="cylinder", seed_noise=0.0, grid_moving=False):
    h = 4.0 / nx
    x0, y0 = -1.0, -2.0
    if kind == "cylinder":
        t = 2 * np.pi / npts * np.arange(npts)
        xb = np.column_stack([0.5 * np.cos(t), 0.5 * np.sin(t)])
        moving = [False]
    elif kind == "plate":
        a = math.radians(30.0)
        xb = np.column_stack([np.linspace(-0.5 * math.cos(a), 0.5 * math.cos(a), npts),
                              np.linspace(0.5 * math.sin(a), -0.5 * math.sin(a), npts)])
        moving = [False]
    else:  # moving plate
        xb = np.column_stack([np.linspace(-0.5, 0.5, npts), np.zeros(npts)])
        moving = [True]
    s = Solver(nx, nx, L, h, x0, y0, Re, dt, xb, [slice(0, npts)], moving, grid_moving=grid_moving)
    if seed_noise:
        rng = np.random.default_rng(12345)
        for lev in range(L):
            s.G[:, lev] = rng.standard_normal(s.gr.ng) * seed_noise * s.gr.hc(lev + 1) ** 2
    G_init = s.G.copy()
    forces = []
    for k in range(nsteps):
        t = dt * k  # t0 + dt (index - 1) after inc_time_index!
        bm = None
        gm = None
        if moving[0]:
            w = 2.0
            bm = [(0.0, 0.1 * math.sin(w * t), 0.0, 0.1 * w * math.cos(w * t), -0.2 * math.sin(w * t),
                   -0.2 * w * math.cos(w * t))]
        if grid_moving:
            gm = (-1.0, 0.0, 0.0, 0.2, 0.1 * math.sin(t), 0.1 * math.cos(t))
        s.advance((1.0, 0.0), bm, gm)
        forces.append(s.fb.sum(axis=0))
    out = dict(nx=nx, L=L, npts=npts, Re=Re, dt=dt, nsteps=nsteps, kind=kind, noise=seed_noise,
               grid_moving=int(grid_moving), xb=xb, Gamma0=G_init, Gamma=s.G, psi=s.psi, q=s.q,
               nonlin1=s.nonlin[0], nonlin2=s.nonlin[1], Fbt=s.Fbt, forces=np.array(forces))
    if s.Binv is not None:
        out["Binv_diag"] = np.diag(s.Binv).copy()
    else:
        out["cg_iters"] = s.cg_iters
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return out


def dst_vectors():
    rng = np.random.default_rng(2026)
    out = {}
    for n in (7, 15, 149, 199, 255, 383, 511):
        x = rng.standard_normal(n)
        out[f"x{n}"] = x
        out[f"y{n}"] = sf.dst(x, type=1)
    x = rng.standard_normal((15, 23))
    out["x2d"] = x
    out["y2d"] = sf.dstn(x, type=1)
    np.savez_compressed(os.path.join(HERE, "dst1_scipy.npz"), **out)


def delta_vectors():
    r = np.linspace(-3.5, 3.5, 701)
    np.savez_compressed(os.path.join(HERE, "delta_h.npz"), r=r, d=delta_h(r, 0.0, 1.0))


if __name__ == "__main__":
    dst_vectors()
    delta_vectors()
    make_case("cyl32_static", 32, 3, 24, 100.0, 0.02, 4)
    make_case("cyl32_noise", 32, 2, 24, 100.0, 0.02, 3, seed_noise=1e-3)
    make_case("plate40_static", 40, 3, 11, 200.0, 0.02, 3, kind="plate")
    make_case("cyl32_movgrid", 32, 3, 24, 100.0, 0.02, 3, grid_moving=True)
    make_case("plate32_moving", 32, 3, 9, 100.0, 0.02, 3, kind="moving")
    print("wrote fixtures to", HERE, file=sys.stderr)

"""Operator-level parity of the CUDA kernels against the CPU oracle: one DST
solve (Δinv, A, Ainv) for every transform-length family, one application of
B, and the precomputed B^-1."""
import numpy as np
import pytest

from fixtures import rel_l2

pytestmark = pytest.mark.gpu


def _lams(orc, prob, op, level):
    nx, ny = prob.grid.base.n
    lam = orc.lap_eigs(nx, ny)
    if op == 0:
        return lam
    hc = prob.grid.gridstep(level)
    den = 2 * prob.fluid.Re * hc ** 2
    if op == 1:
        return 1.0 / (1 - lam * prob.scheme.dt / den)
    return 1 + lam * prob.scheme.dt / den


@pytest.mark.parametrize("n", [32, 40, 48, 64, 150, 200, 256, 384, 512, 1024])
@pytest.mark.parametrize("op", [0, 1, 2])
def test_solve_matches_oracle(ib, orc, n, op):
    prob = ib.configs.small_cylinder(n, 2)
    s = ib.create_solver(ib.State(prob))
    nx, ny = prob.grid.base.n
    rng = np.random.default_rng(n + op)
    b = rng.standard_normal((nx - 1, ny - 1))
    lev = 2 if op else 1
    x = s.diag_solve(op, lev, b)
    ref = orc.lap_inv(nx, ny, _lams(orc, prob, op, lev), b)
    assert rel_l2(x, ref) < 1e-13


@pytest.mark.parametrize("n", [32, 40, 200])
def test_apply_B_and_Binv_match_oracle(ib, orc, n):
    prob = ib.configs.small_cylinder(n, 3)
    g = ib.create_solver(ib.State(prob))
    o = orc.OracleSolver(ib.State(prob))
    m = 2 * prob.bodies.npanel
    rng = np.random.default_rng(n)
    z = rng.standard_normal(m)
    assert rel_l2(g.diag_apply_B(z), o.apply_B(z)) < 1e-12
    assert rel_l2(g.diag_binv(), o.binv()) < 1e-10


@pytest.mark.parametrize("n", [32, 40, 200])
def test_reg_regT_vort2flux_match_oracle(ib, orc, n):
    prob = ib.configs.small_cylinder(n, 3)
    g = ib.create_solver(ib.State(prob))
    o = orc.OracleSolver(ib.State(prob))
    m = 2 * prob.bodies.npanel
    rng = np.random.default_rng(7 + n)
    f = rng.standard_normal(m)
    assert rel_l2(g.diag_reg_rot(f), o.reg_rot(f)) < 1e-14
    q1 = rng.standard_normal(prob.grid.inds.nq)
    assert rel_l2(g.diag_regT(q1), o.regT(q1)) < 1e-14
    G = rng.standard_normal((prob.grid.inds.nGamma, 3))
    ga, pa, qa = g.diag_vort2flux(G)
    gb, pb, qb = o.vort2flux(G)
    assert rel_l2(ga, gb) < 1e-15
    assert rel_l2(pa, pb) < 1e-13
    assert rel_l2(qa, qb) < 1e-12  # curl of a random field differences neighbours

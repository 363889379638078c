"""The FP64 GPU path against the CPU oracle on the configured workloads, at their
full sizes, over the horizons the oracle finishes in about a minute:

  cylinder 200^2 x 3, 157 points, Re 100, dt 0.004   all 500 configured steps
  cylinder 1024^2 x 5, 628 points, seeded noise     the GPU-assembled B and its
      inverse checked against the oracle's B columns and a LAPACK LU inverse,
      then 20 steps with the oracle holding that LU inverse
  plate 1024^2 x 5, 201 points, 30 deg, Re 200      3 steps, the oracle building
      its own B and inverse from scratch
  pitching plate 512^2 x 4, 101 points, Re 500      5 steps of CG to |r| <= 1e-10,
      iteration counts equal within 1 per step

Bars: vorticity (Γ) relative L2 <= 1e-10 and force coefficients <= 1e-9 relative
to the largest (C = 2F / (U^2 L_ref), U = L_ref = 1)."""
import numpy as np
import pytest

from fixtures import rel_l2

pytestmark = pytest.mark.gpu
TOL_GAMMA = 1e-10
TOL_FORCE = 1e-9


def _compare_states(sg, so):
    assert sg.index == so.index
    assert rel_l2(sg.Gamma, so.Gamma) <= TOL_GAMMA, rel_l2(sg.Gamma, so.Gamma)
    assert rel_l2(sg.q, so.q) <= TOL_GAMMA, rel_l2(sg.q, so.q)
    assert rel_l2(sg.psi, so.psi) <= TOL_GAMMA, rel_l2(sg.psi, so.psi)


def _step_both(gpu, cpu, sg, so, nsteps, on_step=None):
    """Advances both solvers, collecting C_D, C_L per step."""
    cg, co = [], []
    for k in range(nsteps):
        gpu.advance_()
        cpu.advance_()
        cg.append(2 * sg.fb.sum(axis=0))
        co.append(2 * so.fb.sum(axis=0))
        if on_step:
            on_step(k)
    gpu.getstate()
    return np.array(cg), np.array(co)


def _assert_forces(cg, co):
    err = np.abs(cg - co).max()
    assert err <= TOL_FORCE * max(1.0, np.abs(co).max()), err


def test_cylinder_200_all_500_steps(ib, orc):
    """src/solver.jl:37-62 driving advance! (:155-190) for the configured 500 steps."""
    prob = ib.configs.cylinder_re100_200()
    sg, so = ib.State(prob), ib.State(prob)
    gpu, cpu = ib.create_solver(sg), orc.OracleSolver(so)
    cg, co = _step_both(gpu, cpu, sg, so, 500)
    _compare_states(sg, so)
    _assert_forces(cg, co)


def test_cylinder_1024_B_inverse_and_20_steps(ib, orc):
    """_Binv_precomputed (src/coupling.jl:187-192) at 1256 x 1256: B as the GPU
    assembles it (the same batched operator, one unit column per call), four of
    its columns against the oracle's B operator (:150-177), the GPU's inverse
    (Gauss-Jordan without pivoting) against B itself and against LAPACK's LU
    inverse (getrf + getri, what LinearAlgebra.inv calls), then the step with the
    oracle holding the LU inverse."""
    prob = ib.configs.cylinder_re100_1024()
    sg = ib.configs.seed_vorticity(ib.State(prob))
    so = ib.configs.seed_vorticity(ib.State(prob))
    gpu = ib.create_solver(sg)
    cpu = orc.OracleSolver(so, timing_only=True)
    n = 2 * prob.bodies.npanel
    B = np.empty((n, n), order="F")
    e = np.zeros(n)
    for c in range(n):
        e[c] = 1.0
        B[:, c] = gpu.diag_apply_B(e)
        e[c] = 0.0
    for c in (0, 311, n // 2 + 17, n - 1):
        e[c] = 1.0
        assert rel_l2(B[:, c], cpu.apply_B(e)) <= 1e-12, c
        e[c] = 0.0
    Bi_gpu = gpu.diag_binv()
    resid = np.abs(B @ Bi_gpu - np.eye(n)).max()
    assert resid <= 1e-8, resid
    Bi_lu = np.linalg.inv(B)
    assert rel_l2(Bi_gpu, Bi_lu) <= 1e-10, rel_l2(Bi_gpu, Bi_lu)
    cpu.set_binv(Bi_lu)
    cg, co = _step_both(gpu, cpu, sg, so, 20)
    _compare_states(sg, so)
    _assert_forces(cg, co)


def test_plate_1024_fp64_against_independent_oracle(ib, orc):
    """The configured mixed-precision workload's geometry in FP64 (flat plate of
    chord 1 at 30 deg, Re 200, 1024^2 x 5, 201 points, dt 0.001, from rest); the
    oracle builds B and its LU inverse itself."""
    prob = ib.configs.plate_aoa30_1024()
    sg, so = ib.State(prob), ib.State(prob)
    gpu, cpu = ib.create_solver(sg), orc.OracleSolver(so)
    cg, co = _step_both(gpu, cpu, sg, so, 3)
    _compare_states(sg, so)
    _assert_forces(cg, co)


def test_pitching_plate_512_cg_iterations(ib, orc):
    """The moving-body workload (512^2 x 4, 101-point plate pitching and plunging
    at k = 0.55, Re 500, dt 0.002): B applied inside CG each iteration
    (_Binv_iterative, src/coupling.jl:194-202), CG to |r| <= 1e-10 from the
    previous solution; iteration counts equal within 1 at every step."""
    cgopt = dict(reltol=0.0, abstol=1e-10, maxiter=5000)
    prob = ib.configs.pitching_plate(0.55)
    sg, so = ib.State(prob), ib.State(prob)
    gpu = ib.GpuCnabSolver(sg, cg=cgopt)
    cpu = orc.OracleSolver(so, cg=cgopt)
    its = []

    def count(k):
        its.append((gpu.info().last_cg_iters, cpu.last_cg_iters()))

    cg, co = _step_both(gpu, cpu, sg, so, 5, count)
    for ig, io in its:
        assert abs(ig - io) <= 1, its
    _compare_states(sg, so)
    _assert_forces(cg, co)

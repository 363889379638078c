"""Ensembles (ibpm_ensemble_*): independent cases stepped together must give
each case exactly the results of stepping it alone; and multi-step calls must
give the results of single steps when the host callbacks vary in time (the
per-step parameters travel through pinned staging that is reused only after the
copies that read it have run)."""
import math
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(ib):
    # three seeded cases of two widths, cylinders and plates, spacing 0.04
    return ib.configs.ensemble_cases(3, seed=7, h=0.04, widths=(64, 96), ny=64)


def test_ensemble_matches_cases_stepped_alone(ib):
    probs = _cases(ib)
    precs = ["fp64", "fp32", "fp64"]
    alone = [ib.GpuCnabSolver(ib.State(p), precision=pr) for p, pr in zip(probs, precs)]
    for s in alone:
        s.advance_many(6)
    together = [ib.GpuCnabSolver(ib.State(p), precision=pr) for p, pr in zip(probs, precs)]
    ens = ib.Ensemble(together)
    ens.advance_(4)
    ens.advance_(2)
    for a, b in zip(alone, together):
        sa, sb = a.getstate(), b.getstate()
        assert sa.index == sb.index == 6
        assert np.array_equal(sa.Gamma, sb.Gamma)
        assert np.array_equal(sa.q, sb.q)
        assert np.array_equal(a.total_force(), b.total_force())
        assert np.array_equal(sa.fb, sb.fb)


def test_cases_destroyed_before_their_ensemble(ib):
    probs = ib.configs.ensemble_cases(3, seed=7, h=0.04, widths=(64,), ny=64)
    sol = [ib.GpuCnabSolver(ib.State(p), precision="fp32") for p in probs]
    ens = ib.Ensemble(sol)
    assert ens.groups() == (1, 3)
    ens.advance_(2)
    sol[0].close()  # the group's first case goes first
    with pytest.raises(ib._abi.IbpmError):
        ens.advance_(1)
    ens.close()  # copies the live cases back; never touches the destroyed one
    for s in sol[1:]:
        s.advance_()
        assert s.getstate().index == 3


def test_interpreter_exit_with_a_live_ensemble():
    # objects at module level with a module-level function form one reference
    # cycle at exit, whose finalizers run in allocation order: every solver's
    # before the ensemble's
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {os.path.join(root, "tests")!r})
        from conftest import load_package
        ib = load_package()
        probs = ib.configs.ensemble_cases(3, seed=7, h=0.04, widths=(64, 96), ny=64)
        sol = [ib.GpuCnabSolver(ib.State(p), precision="fp32") for p in probs]
        ens = ib.Ensemble(sol)
        def step():
            ens.advance_(2)
        step()
        print("stepped")
    """)
    r = subprocess.run([sys.executable, "-X", "faulthandler", "-c", script], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "stepped" in r.stdout, r.stderr[-2000:]


def _gusty_cylinder(ib):
    def gust(t):
        return (1.0 + 0.5 * math.sin(40.0 * t), 0.2 * math.cos(25.0 * t))

    h = 0.04
    fluid = ib.Fluid(grid=ib.fluid_grid(h=h, xlims=(-1.0, 1.56), ylims=(-1.28, 1.28), nlevel=2), Re=100.0,
                     freestream_vel=gust)
    panels = ib.Curves.partition(ib.Curves.Circle(r=0.5, center=(0.0, 0.0)), 79)
    return ib.Problem(fluid=fluid, bodies=ib.Bodies(cyl=ib.StaticBody(panels)), scheme=ib.CNAB(dt=0.008))


def test_multi_step_call_with_time_varying_freestream(ib):
    prob = _gusty_cylinder(ib)
    one = ib.GpuCnabSolver(ib.State(prob))
    for _ in range(12):
        one.advance_()
    many = ib.GpuCnabSolver(ib.State(prob))
    many.advance_many(12)
    assert np.array_equal(one.getstate().Gamma, many.getstate().Gamma)
    assert np.array_equal(one.total_force(), many.total_force())


def _gusty_cases(ib, n, seed, width):
    """n seeded cylinders and plates of one shape (a batched group: width x 64
    cells at h 0.04, 3 levels) with different Reynolds numbers and bodies, in a
    time-varying freestream."""
    def gust(t):
        return (1.0 + 0.3 * math.sin(30.0 * t), 0.1 * math.cos(20.0 * t))

    probs = ib.configs.ensemble_cases(n, seed=seed, h=0.04, widths=(width,), ny=64)
    for p in probs:
        p.fluid.freestream_vel = gust
    return probs


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batched_group_matches_cases_stepped_alone(ib, prec):
    """18 cases of one shape form one batched group (18 >= 16 fields also takes
    the wide Y-pass blocks) and two more of another width a second group.
    Every case's state and forces equal stepping it alone, bit for bit,
    across calls of several steps with a time-varying freestream; after the
    ensemble is destroyed each case steps on alone from where it was."""
    probs = _gusty_cases(ib, 18, 11, 96) + _gusty_cases(ib, 2, 5, 64)
    alone = [ib.GpuCnabSolver(ib.State(p), precision=prec) for p in probs]
    for s in alone:
        s.advance_many(7)
    together = [ib.GpuCnabSolver(ib.State(p), precision=prec) for p in probs]
    ens = ib.Ensemble(together)
    assert ens.groups() == (2, 20)
    ens.advance_(3)
    ens.advance_(1)
    ens.advance_(3)
    for a, b in zip(alone, together):
        sa, sb = a.getstate(), b.getstate()
        assert sa.index == sb.index == 7
        assert np.array_equal(sa.Gamma, sb.Gamma)
        assert np.array_equal(sa.q, sb.q)
        assert np.array_equal(sa.psi, sb.psi)
        assert np.array_equal(sa.nonlin[0], sb.nonlin[0]) and np.array_equal(sa.nonlin[1], sb.nonlin[1])
        assert np.array_equal(a.total_force(), b.total_force())
    ens.close()
    for a, b in zip(alone, together):
        a.advance_many(2)
        b.advance_many(2)
        assert np.array_equal(a.getstate().Gamma, b.getstate().Gamma)
        assert np.array_equal(a.total_force(), b.total_force())


def test_grouping_can_be_disabled(ib, monkeypatch):
    probs = _gusty_cases(ib, 3, 13, 96)
    monkeypatch.setenv("IBPM_ENSEMBLE_BATCH", "0")
    ens = ib.Ensemble([ib.GpuCnabSolver(ib.State(p)) for p in probs])
    assert ens.groups() == (0, 0)
    ens.advance_(2)
    assert np.isfinite(ens.total_forces()).all()

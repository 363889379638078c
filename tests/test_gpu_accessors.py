"""Device-side output accessors (ibpm_get_field) against the host mirror of the
reference's vorticity!, x_velocity!, y_velocity! (src/problem.jl:715-866)
applied to the full state: same values, bit for bit, one level at a time."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_accessors_match_host(ib):
    prob = ib.configs.small_cylinder(48, 3)
    s = ib.GpuCnabSolver(ib.configs.seed_vorticity(ib.State(prob)))
    s.advance_many(3)
    st = s.getstate()
    w, u, v = ib.vorticity(st), ib.x_velocity(st), ib.y_velocity(st)
    for lev in (1, 2, 3):
        assert np.array_equal(s.vorticity(lev), w[..., lev - 1])
        assert np.array_equal(s.x_velocity(lev), u[..., lev - 1])
        assert np.array_equal(s.y_velocity(lev), v[..., lev - 1])
    with pytest.raises(ib._abi.IbpmError, match="level out of range"):
        s.vorticity(4)


def test_accessors_before_the_first_step(ib):
    """State(prob) has q0 = 0 until the first step (problem.jl:640-665)."""
    s = ib.GpuCnabSolver(ib.configs.seed_vorticity(ib.State(ib.configs.small_cylinder(48, 2))))
    st = s.getstate()
    assert np.array_equal(s.x_velocity(1), ib.x_velocity(st)[..., 0])
    assert np.array_equal(s.vorticity(2), ib.vorticity(st)[..., 1])

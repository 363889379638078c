"""The premise of the preconditioned CG start, checked on the CPU oracle.

The preconditioned mode (IBPM_WS_PRECONDITIONED) preconditions the force solve's
CG with B^-1 of a few steps back.  The reference's own operator B
(src/coupling.jl:150-177) is assembled here column by column from the oracle's
apply_B for a small pitching plate, before and after the body moves, and the
test checks that the stale inverse clusters the spectrum of the new B near 1 and
that CG preconditioned by it converges in a handful of iterations where plain CG
needs many.  The CG here is IterativeSolvers' iteration (with Pl for the
preconditioned one) and stops by the reference's rule ||r|| <= abstol."""
import numpy as np


def _assemble(s, n):
    return np.stack([s.apply_B(np.eye(n)[k]) for k in range(n)], axis=1)


def _cg(B, b, x0, Minv=None, abstol=1e-10, maxiter=2000):
    x = x0.copy()
    r = b - B @ x
    u = np.zeros_like(r)
    rho_prev = 1.0
    for it in range(maxiter):
        if np.linalg.norm(r) <= abstol:
            return it, x
        z = Minv @ r if Minv is not None else r
        rho = r @ z
        u = z + (rho / rho_prev) * u
        rho_prev = rho
        c = B @ u
        alpha = rho / (u @ c)
        x = x + alpha * u
        r = r - alpha * c
    return maxiter, x


def test_stale_inverse_preconditions_cg(ib, orc):
    prob = ib.configs.pitching_plate(0.55, h=0.04, n=128, nlevel=3, npts=26, dt=0.004)
    s = orc.OracleSolver(ib.State(prob))
    n = 2 * 26
    for _ in range(10):
        s.advance_()
    Minv = np.linalg.inv(_assemble(s, n))
    for _ in range(4):
        s.advance_()
    B = _assemble(s, n)
    lam = np.linalg.eigvals(Minv @ B)
    assert np.abs(lam - 1).max() < 0.2, np.abs(lam - 1).max()
    rng = np.random.default_rng(7)
    b = B @ (1e-2 * rng.normal(size=n))
    it_plain, x_plain = _cg(B, b, Minv @ b)
    it_pre, x_pre = _cg(B, b, Minv @ b, Minv)
    assert it_pre <= 8 and it_plain >= 5 * it_pre, (it_pre, it_plain)
    # both meet the same residual, so they agree to within the conditioning of B
    x = np.linalg.solve(B, b)
    assert np.linalg.norm(x_pre - x) <= 1e-6 * np.linalg.norm(x)

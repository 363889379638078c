"""The tensor-core DST-I passes (csrc/tc_dst.cu) and the preconditioner they build.

A 2D solve x = S(m ⊙ S(b)) (src/fluid.jl:145-166 with FFTW's RODFT00 as S) runs
as four dense passes D = S X on tcgen05 with BF16 operands and FP32
accumulation, each pass two half-length products by the transform's
even/odd symmetry.  `_emulate` restates that arithmetic in numpy (the same
splits, roundings and pass order, with round-to-nearest FP32 sums): with one product the
GPU result must sit on the emulation, far closer than either sits to the FP64
solve; with three, whose low parts the accumulator's own rounding reaches, within
a small factor of the emulation's error.  The preconditioned moving-body modes then assemble B with these solves:
CG still stops at the same tolerance, so forces agree with the FP64 rebuild to
that tolerance, and the inverse preconditions B well."""
import numpy as np
import pytest
import scipy.fft as sf

pytestmark = pytest.mark.gpu

CG = dict(reltol=0.0, abstol=1e-10, maxiter=5000)


def _bf16(x):
    x = np.asarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def _split(v):
    h = _bf16(v)
    return h, _bf16(np.asarray(v, np.float64) - h)


def _uv(X, axis_len):
    """u (j = 1 .. P/2) and v (j = 1 .. P/2 - 1) of the lines X[line][j - 1]."""
    P = axis_len
    h = P // 2
    j = np.arange(1, h)
    u = np.concatenate([X[:, j - 1] + X[:, P - j - 1], X[:, h - 1:h]], axis=1)
    v = X[:, j - 1] - X[:, P - j - 1]
    return u, v


def _emulate(b2, mult, nprod):
    """The four passes on (P-1)^2 field b2 [y][x] with multipliers mult [ky][kx]:
    each pass y_k = sum_j S[k][j] u_j (odd k) or v_j (even k) with BF16 operands
    (split into hi + lo for three products) and FP32 sums, u, v of the lines
    formed in FP64 from the input and in FP32 between passes."""
    m = b2.shape[0]
    P = m + 1
    h = P // 2
    ko, ke = np.arange(1, P, 2), np.arange(2, P, 2)
    Ao = 2 * np.sin(np.pi * np.outer(ko, np.arange(1, h + 1)) / P)
    Ae = 2 * np.sin(np.pi * np.outer(ke, np.arange(1, h)) / P)
    Aoh, Aol = _split(Ao)
    Aeh, Ael = _split(Ae)

    def prod(Ah, Al, X):  # X: FP64 or FP32 values of the lines' u or v
        Xh, Xl = _split(X)
        D = Ah @ Xh.T
        if nprod == 3:
            D = D + Ah @ Xl.T + Al @ Xh.T
        return D.astype(np.float32)

    def dpass(X):  # X[line][position], positions 1 .. P-1; returns D[k - 1][line]
        u, v = _uv(X, P)
        D = np.zeros((m, X.shape[0]), np.float32)
        D[ko - 1] = prod(Aoh, Aol, u)
        D[ke - 1] = prod(Aeh, Ael, v)
        return D

    D1 = dpass(b2.astype(np.float64))             # [kx][y]
    D2 = (dpass(D1) * mult).astype(np.float32)    # [ky][kx]
    D4 = dpass(dpass(D2))                         # [x][ky] -> [y][x]
    return D4.astype(np.float64)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _plate(ib, n=256):
    prob = ib.configs.pitching_plate(0.5, h=0.02, n=n, nlevel=3, npts=51, dt=0.004)
    return ib.GpuCnabSolver(ib.State(prob), cg=CG)


@pytest.mark.parametrize("n", [256, 512])
def test_tensor_core_solve_follows_its_arithmetic(ib, n):
    """Δinv and Ainv (level 2) of a seeded field through ibpm_diag_solve ops 3..8."""
    s = _plate(ib, n)
    m = n - 1
    rng = np.random.default_rng(n)
    b = rng.normal(size=(m, m))  # [y][x]
    i = np.arange(1, n)
    lam = -2 * (np.cos(np.pi * i[None, :] / n) + np.cos(np.pi * i[:, None] / n) - 2)  # [ky][kx]
    scale = 1.0 / (4 * n * n)
    hc = s.state.prob.fluid.grid.gridstep(2)
    c = s.state.prob.scheme.dt / (2 * s.state.prob.fluid.Re * hc * hc)
    mults = {0: scale / lam, 2: scale / (1 + lam * c)}
    bf = b.T.reshape(-1, order="F")  # column-major (x fastest) field of the ABI
    for op, mult in mults.items():
        exact = sf.dstn(sf.dstn(b, type=1) * mult, type=1)
        x64 = s.diag_solve(op, 2, bf).reshape(m, m, order="F").T
        assert _rel(x64, exact) <= 1e-12
        for nprod, bar in ((1, 1e-2), (3, 2e-5)):
            emu = _emulate(b, mult.astype(np.float32), nprod)
            xtc = s.diag_solve(op + (3 if nprod == 1 else 6), 2, bf).reshape(m, m, order="F").T
            e_emu, e_gpu = _rel(emu, exact), _rel(xtc, exact)
            print(f"n={n} op={op} products={nprod}: error {e_gpu:.3e} (emulated {e_emu:.3e}), "
                  f"from the emulation {_rel(xtc, emu):.3e}")
            assert e_gpu <= bar, (op, nprod, e_gpu)
            if nprod == 1:
                # the BF16 roundings dominate: the GPU sits on the emulated arithmetic
                # (a value at a rounding tie may round the other way after a
                # different FP32 summation order)
                assert abs(e_gpu - e_emu) <= 0.02 * e_emu, (op, nprod, e_gpu, e_emu)
                assert _rel(xtc, emu) <= 0.35 * e_emu, (op, nprod, _rel(xtc, emu), e_emu)
            else:
                # the tensor cores' FP32 accumulation is not round-to-nearest, which
                # the split products expose; the error stays at the emulated scale
                assert e_gpu <= 4 * e_emu, (op, nprod, e_gpu, e_emu)


@pytest.mark.parametrize("products", [1, 3])
def test_tensor_core_rebuild_preconditions_cg(ib, products):
    """The preconditioned mode with B assembled on the tensor cores: the inverse
    of a rebuild step against B assembled in FP64 (diag_apply_B), and 24 steps
    whose forces match the FP64 rebuild's to the CG tolerance with about as many
    iterations."""
    runs = {}
    for prod in (0, products):
        s = _plate(ib)
        s.set_warm_start(None, mode="preconditioned", depth=8)
        s.set_rebuild_transform(prod)
        it = []
        for k in range(24):
            s.advance_()
            it.append(s.info().last_cg_iters)
            if k == 16 and prod:  # a rebuild step: Binv is this step's
                n = 2 * s.state.prob.bodies.npanel
                B = np.stack([s.diag_apply_B(np.eye(n)[q]) for q in range(n)], axis=1)
                lam = np.linalg.eigvals(s.diag_binv() @ B)
                spread = np.abs(lam - 1).max()
                assert spread <= (0.1 if products == 1 else 1e-3), spread
        runs[prod] = (np.asarray(it), s.total_force().copy())
        del s
    (i0, f0), (it, f) = runs[0], runs[products]
    assert np.abs(f - f0).max() <= 1e-6 * np.abs(f0).max()
    assert it.mean() <= i0.mean() + (2 if products == 1 else 0.5), (it, i0)


@pytest.mark.parametrize("products", [1, 3])
def test_tensor_core_preconditioner_on_the_moving_plate(ib, products):
    """The configured moving-body workload (512^2 x 4, 101-point plate, k = 0.55)
    with the extrapolated preconditioned start rebuilt every 8th step, over the
    160 steps the bench runs: every step converges in a handful of iterations (the symmetric part of the
    tensor-core inverse keeps CG's preconditioner symmetric) and the forces are
    the FP64 rebuild's to the CG tolerance."""
    runs = {}
    for prod in (0, products):
        s = ib.GpuCnabSolver(ib.State(ib.configs.pitching_plate(0.55)), cg=CG)
        s.set_warm_start(None, mode="preconditioned_extrapolated", depth=8)
        s.set_rebuild_transform(prod)
        it = []
        for _ in range(160):
            s.advance_()
            it.append(s.info().last_cg_iters)
        runs[prod] = (np.asarray(it), s.total_force().copy())
        print(f"products {prod}: CG iterations mean {np.mean(it):.2f}, max {np.max(it)}")
        del s
    (i0, f0), (it, f) = runs[0], runs[products]
    assert it.max() <= 40, it
    assert np.abs(f - f0).max() <= 1e-6 * np.abs(f0).max()


def test_tensor_core_rebuild_eager_matches_graph(ib):
    """With profiling on the rebuild runs without its graph: the same iterations
    and forces, and the tensor-core class is timed."""
    out = {}
    for eager in (False, True):
        s = _plate(ib)
        s.set_warm_start(None, mode="preconditioned_extrapolated", depth=4)
        s.set_rebuild_transform(3)
        if eager:
            s.profile(True)
        it = []
        for _ in range(9):
            s.advance_()
            it.append(s.info().last_cg_iters)
        if eager:
            n, ms, _ = s.profile_read("tcdst")
            assert n > 0 and ms > 0
        out[eager] = (it, s.total_force().copy())
        del s
    assert out[False][0] == out[True][0]
    assert np.abs(out[False][1] - out[True][1]).max() <= 1e-13 * np.abs(out[False][1]).max()


def test_tensor_core_rebuild_errors(ib):
    s = _plate(ib)
    with pytest.raises(Exception):
        s.set_rebuild_transform(2)
    prob = ib.configs.pitching_plate(0.5, h=0.04, n=128, nlevel=3, npts=26, dt=0.004)
    s2 = ib.GpuCnabSolver(ib.State(prob), cg=CG)
    with pytest.raises(Exception):
        s2.set_rebuild_transform(3)  # 128 x 128 is not a tensor-core size
    s2.set_rebuild_transform(0)

"""The learned CG warm start: its network's CUDA kernels against the CPU oracle
(oracle/warmstart_net.py), training, and what it changes in the moving-body
force solve.

The reference starts cg! from the previous F~b (src/coupling.jl:194-202); the
warm start changes only that initial guess, so every mode must reach the same
forces to the CG tolerance, and the tests compare iteration counts."""
import numpy as np
import pytest

from oracle import warmstart_net as wn

pytestmark = pytest.mark.gpu

ARCH = dict(cin=10, width=64, kernel=5, layers=4, cout=2)
CG = dict(reltol=0.0, abstol=1e-10, maxiter=5000)


def _net(ib, seed=1):
    return ib.WarmStartNet(width=ARCH["width"], kernel=ARCH["kernel"], layers=ARCH["layers"], seed=seed)


def _random_case(ib, net, B=6, N=101, seed=0):
    rng = np.random.default_rng(seed)
    net.set_normalisation(rng.normal(size=10), rng.uniform(0.5, 2, 10), rng.normal(size=2), rng.uniform(0.5, 2, 2))
    x = rng.normal(size=(B, 10, N)).astype(np.float32)
    t = rng.normal(size=(B, 2, N)).astype(np.float32)
    shapes = wn.layer_shapes(**{k: ARCH[k] for k in ("cin", "width", "kernel", "layers", "cout")})
    norm = [a.astype(np.float64) for a in net.normalisation()]
    return x, t, shapes, norm


def test_forward_matches_oracle(ib):
    net = _net(ib)
    x, _, shapes, norm = _random_case(ib, net)
    y = net.forward(x)
    yr = wn.predict(net.get_params().astype(np.float64), shapes, norm, x.astype(np.float64))
    assert np.abs(y - yr).max() <= 1e-5 * np.abs(yr).max()


def test_gradient_matches_oracle(ib):
    """FP32 kernels (fixed reduction order) against the float64 oracle: 1e-5 relative."""
    net = _net(ib)
    x, t, shapes, norm = _random_case(ib, net, B=5, N=37, seed=3)
    loss, g = net.loss_grad(x, t)
    lr, gr = wn.loss_grad(net.get_params().astype(np.float64), shapes, norm, x.astype(np.float64),
                          t.astype(np.float64))
    assert abs(loss - lr) <= 1e-5 * abs(lr)
    assert np.linalg.norm(g - gr) <= 1e-5 * np.linalg.norm(gr)
    # the gradient is exact for the stated loss: a step along -g lowers it
    p = net.get_params()
    net.set_params(p - 1e-3 * g / np.linalg.norm(g))
    assert net.loss_grad(x, t)[0] < loss


def test_training_lowers_the_loss_and_is_deterministic(ib):
    rng = np.random.default_rng(5)
    x = rng.normal(size=(256, 10, 33)).astype(np.float32)
    # a smooth local linear map of the inputs the network can represent
    t = np.stack([x[:, 0] + 0.5 * np.roll(x[:, 1], 1, axis=1), x[:, 2] - x[:, 3]], axis=1).astype(np.float32)
    runs = []
    for _ in range(2):
        net = _net(ib, seed=11)
        net.fit_normalisation(x, t)
        losses = net.train(x, t, epochs=60, batch=32, lr=2e-3, seed=3)
        runs.append((losses, net.get_params()))
    losses, p = runs[0]
    assert losses[-1] < 0.05 * losses[0], losses[[0, -1]]
    assert np.array_equal(p, runs[1][1]) and np.array_equal(losses, runs[1][0])


def _plate(ib, k):
    prob = ib.configs.pitching_plate(k, h=0.04, n=128, nlevel=3, npts=26, dt=0.004)
    return ib.GpuCnabSolver(ib.State(prob), cg=CG)


def _iters(s, n):
    it = []
    for _ in range(n):
        s.advance_()
        it.append(s.info().last_cg_iters)
    return np.asarray(it)


def test_every_start_reaches_the_same_forces(ib):
    forces, iters = {}, {}
    for mode in ("previous", "extrapolated", "projected"):
        s = _plate(ib, 0.5)
        if mode != "previous":
            s.set_warm_start(None, mode=mode, depth=8)
        iters[mode] = _iters(s, 40)
        forces[mode] = s.total_force().copy()
        if mode == "projected":
            assert s.info().warm_start_coef[0] >= 2  # directions kept by the projection
        del s
    f0 = forces["previous"]
    for mode in ("extrapolated", "projected"):
        assert np.abs(forces[mode] - f0).max() <= 1e-6 * np.abs(f0).max(), mode
    assert iters["extrapolated"][10:].mean() < iters["previous"][10:].mean()
    assert iters["projected"][10:].mean() < iters["extrapolated"][10:].mean()


def test_direct_start_matches_the_reference_start(ib):
    """B assembled and inverted on the GPU each step (or every 4th): CG starts at
    B^-1 b, so it needs no iterations on a rebuild step, and every start reaches
    the forces of the reference's start to the CG tolerance.  Between rebuilds
    the inverse of a few steps back gives a guess no worse than the reference's
    (B moves with the body, so it saves only a few iterations)."""
    runs = {}
    for mode, depth in (("previous", 8), ("direct", 1), ("direct", 4)):
        s = _plate(ib, 0.5)
        if mode != "previous":
            s.set_warm_start(None, mode=mode, depth=depth)
        runs[(mode, depth)] = (_iters(s, 24), s.total_force().copy())
        del s
    it0, f0 = runs[("previous", 8)]
    for key in (("direct", 1), ("direct", 4)):
        it, f = runs[key]
        assert np.abs(f - f0).max() <= 1e-6 * np.abs(f0).max(), key
    assert runs[("direct", 1)][0].max() <= 1
    it4 = runs[("direct", 4)][0]
    assert it4[::4].max() <= 1  # rebuild steps
    assert it4[8:].mean() <= 1.05 * it0[8:].mean()


def test_preconditioned_cg_with_a_periodic_inverse(ib):
    """CG preconditioned by B^-1 of the last rebuild (every 8th step): a few
    iterations between rebuilds, and the forces of the reference's unpreconditioned
    CG to its tolerance."""
    runs = {}
    for mode in ("previous", "preconditioned"):
        s = _plate(ib, 0.5)
        if mode != "previous":
            s.set_warm_start(None, mode=mode, depth=8)
        runs[mode] = (_iters(s, 24), s.total_force().copy())
        del s
    (it0, f0), (it, f) = runs["previous"], runs["preconditioned"]
    assert np.abs(f - f0).max() <= 1e-6 * np.abs(f0).max()
    assert it[::8].max() <= 1  # rebuild steps start at B^-1 b of their own B
    assert it.max() <= 12 and it.mean() <= 0.1 * it0.mean(), (it, it0.mean())


def test_preconditioned_extrapolated_start_saves_iterations(ib):
    """The preconditioned mode started from B^-1 b plus the stale error F - B^-1 b
    extrapolated from the last steps' (rebuild every 16th step): fewer CG
    iterations between rebuilds than from B^-1 b alone, the same at rebuild
    steps, and the reference start's forces to the CG tolerance."""
    runs = {}
    for mode in ("previous", "preconditioned", "preconditioned_extrapolated"):
        s = _plate(ib, 0.5)
        if mode != "previous":
            s.set_warm_start(None, mode=mode, depth=16)
        runs[mode] = (_iters(s, 48), s.total_force().copy())
        del s
    (_, f0), (itp, _), (ite, fe) = runs["previous"], runs["preconditioned"], runs["preconditioned_extrapolated"]
    assert np.abs(fe - f0).max() <= 1e-6 * np.abs(f0).max()
    assert ite[::16].max() <= 1
    between = [k for k in range(len(ite)) if k % 16 >= 3]  # three stale errors known
    assert ite[between].mean() < itp[between].mean() - 0.5, (ite, itp)


def test_direct_and_preconditioned_eager_match_graphs(ib):
    """With kernel profiling on, steps run eagerly: the B^-1 rebuild without its
    graph and CG as a host loop.  Both modes give the graph path's iteration
    counts and forces."""
    out = {}
    for mode in ("direct", "preconditioned", "preconditioned_extrapolated"):
        for eager in (False, True):
            s = _plate(ib, 0.5)
            s.set_warm_start(None, mode=mode, depth=4)
            if eager:
                s.profile(True)
            out[(mode, eager)] = (_iters(s, 10), s.total_force().copy())
            del s
    for mode in ("direct", "preconditioned", "preconditioned_extrapolated"):
        (ig, fg), (ie, fe) = out[(mode, False)], out[(mode, True)]
        assert np.array_equal(ig, ie), (mode, ig, ie)
        assert np.abs(fe - fg).max() <= 1e-13 * np.abs(fg).max(), mode


def test_direct_start_inverts_the_current_B(ib):
    """After a step the direct start's inverse is the inverse of B at the step's
    body position, B assembled here column by column through diag_apply_B."""
    s = _plate(ib, 0.5)
    s.set_warm_start(None, mode="direct", depth=1)
    for _ in range(3):
        s.advance_()
    n = 2 * s.state.prob.bodies.npanel
    B = np.stack([s.diag_apply_B(np.eye(n)[k]) for k in range(n)], axis=1)
    Binv = s.diag_binv()
    assert np.abs(Binv @ B - np.eye(n)).max() <= 1e-8


def test_every_start_keeps_the_reference_relative_tolerance(ib):
    """With the reference's CG options (reltol 1e-12 of the residual at its start
    F1, abstol 0) every start stops at the tolerance the reference's start sets,
    so a better start needs fewer iterations, never more, and all reach the same
    forces."""
    cg = dict(reltol=1e-12, abstol=0.0, maxiter=5000)
    res = {}
    for mode, depth in (("previous", 8), ("extrapolated", 8), ("projected", 8), ("direct", 1), ("preconditioned", 8)):
        prob = ib.configs.pitching_plate(0.5, h=0.04, n=128, nlevel=3, npts=26, dt=0.004)
        s = ib.GpuCnabSolver(ib.State(prob), cg=cg)
        if mode != "previous":
            s.set_warm_start(None, mode=mode, depth=depth)
        it = _iters(s, 30)
        res[mode] = (it[10:].mean(), s.total_force().copy())
        del s
    it0, f0 = res["previous"]
    for mode, (it, f) in res.items():
        assert it <= 1.02 * it0 + 1, (mode, it, it0)
        assert np.abs(f - f0).max() <= 1e-7 * np.abs(f0).max(), mode
    assert res["direct"][0] <= 2 and res["preconditioned"][0] <= 10


def test_learned_warm_start_on_a_held_out_frequency(ib, capsys):
    """Trained on samples of k = 0.3 and 0.7, run at k = 0.5.  The learned start
    includes the extrapolation step, so it must use fewer CG iterations than the
    reference's start and no more than extrapolation alone; the printed numbers
    show how much of the gain the network itself adds."""
    xs, ts = [], []
    for k in (0.3, 0.7):
        s = _plate(ib, k)
        x, t, _ = ib.warmstart.collect_samples(s, 120, skip=30)
        xs.append(x)
        ts.append(t)
        del s
    X, T = np.concatenate(xs), np.concatenate(ts)
    net = _net(ib, seed=2026)
    net.fit_normalisation(X, T)
    net.train(X, T, epochs=150, batch=32, lr=1e-3)
    net.train(X, T, epochs=100, batch=32, lr=2e-4, seed=8)
    res = {}
    for mode in ("previous", "extrapolated", "learned"):
        s = _plate(ib, 0.5)
        if mode != "previous":
            s.set_warm_start(net if mode == "learned" else None, mode=mode)
        it = _iters(s, 100)
        if mode == "learned":
            f, t, p = s.warm_start_sample(prediction=True)
            # the step used the network's own prediction for these features
            ph = net.forward(f[None])[0]
            assert np.abs(p - ph).max() <= 1e-4 * np.abs(ph).max()
        res[mode] = it[30:].mean()
        del s
    with capsys.disabled():
        print(f"\nCG iterations at held-out k=0.5: previous {res['previous']:.1f}, extrapolated "
              f"{res['extrapolated']:.1f}, learned {res['learned']:.1f}")
    assert res["learned"] < 0.97 * res["previous"]
    assert res["learned"] <= 1.02 * res["extrapolated"]


def test_warm_start_errors(ib):
    static = ib.GpuCnabSolver(ib.State(ib.configs.small_cylinder(48, 2)))
    with pytest.raises(ib._abi.IbpmError, match="moving bodies"):
        static.set_warm_start(None, mode="extrapolated")
    s = _plate(ib, 0.5)
    with pytest.raises(ib._abi.IbpmError, match="needs a network"):
        s.set_warm_start(None, mode="learned")
    with pytest.raises(ib._abi.IbpmError, match="depth"):
        s.set_warm_start(None, mode="projected", depth=17)
    s.advance_()
    with pytest.raises(ib._abi.IbpmError, match="extrapolated or learned"):
        s.warm_start_sample()
    wrong = ib.WarmStartNet(cin=4, width=8, layers=2)
    with pytest.raises(ib._abi.IbpmError, match="10 feature channels"):
        s.set_warm_start(wrong)
    with pytest.raises(ib._abi.IbpmError, match="rebuild interval"):
        s.set_warm_start(None, mode="direct", depth=0)
    prob = ib.configs.pitching_plate(0.5, h=0.04, n=128, nlevel=3, npts=26, dt=0.004)
    s32 = ib.GpuCnabSolver(ib.State(prob), cg=CG, precision="fp32")
    with pytest.raises(ib._abi.IbpmError, match="FP64 engine"):
        s32.set_warm_start(None, mode="direct")

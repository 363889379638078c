"""CPU checks of the warm-start network's oracle (oracle/warmstart_net.py):
its gradients against central finite differences, and the parameter layout the
CUDA network uses (per layer W [out][in][kernel], then b [out])."""
import numpy as np

from oracle import warmstart_net as wn


def _case(seed=3, cin=4, width=6, kernel=5, layers=3, cout=2, B=3, N=11):
    rng = np.random.default_rng(seed)
    shapes = wn.layer_shapes(cin, width, kernel, layers, cout)
    p = rng.normal(0, 0.4, wn.num_params(cin, width, kernel, layers, cout))
    norm = (rng.normal(0, 1, cin), rng.uniform(0.5, 2, cin), rng.normal(0, 1, cout), rng.uniform(0.5, 2, cout))
    x = rng.normal(0, 1, (B, cin, N))
    t = rng.normal(0, 1, (B, cout, N))
    return p, shapes, norm, x, t


def test_parameter_count_of_the_warm_start_network():
    # 10 feature channels, width 64, kernel 5, 4 layers, 2 outputs
    assert wn.num_params(10, 64, 5, 4, 2) == 10 * 64 * 5 + 64 + 2 * (64 * 64 * 5 + 64) + 64 * 2 * 5 + 2 == 44994


def test_gradient_matches_central_differences():
    p, shapes, norm, x, t = _case()
    loss, g = wn.loss_grad(p, shapes, norm, x, t)
    rng = np.random.default_rng(0)
    idx = rng.choice(p.size, 60, replace=False)
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (wn.loss_grad(pp, shapes, norm, x, t)[0] - wn.loss_grad(pm, shapes, norm, x, t)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_zero_padding_and_receptive_field():
    # with one layer of kernel 5, output point n depends on inputs n-2..n+2 only
    p, shapes, norm, x, t = _case(layers=1, cout=1, cin=1, width=1)
    y0, _ = wn.forward(p, shapes, norm, x)
    x2 = x.copy()
    x2[:, :, 8] += 1.0
    y1, _ = wn.forward(p, shapes, norm, x2)
    changed = np.nonzero(np.abs(y1 - y0).max(axis=(0, 1)) > 0)[0]
    assert changed.tolist() == [6, 7, 8, 9, 10]

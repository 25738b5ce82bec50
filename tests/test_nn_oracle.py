"""The warm-start network's CPU oracle checks itself: its analytic
gradients (the backward pass the device mirrors) against central finite
differences of its forward pass, on every layer of the encoder-decoder."""
import numpy as np

from atlaswerks_b200.warmstart import LAYERS, n_parameters
from oracle import nn_oracle as O


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    W = {n: rng.normal(0, 0.1, (co, t, ci)).astype(np.float32) for n, ci, co, t in LAYERS}
    B = {n: rng.normal(0, 0.01, co).astype(np.float32) for n, ci, co, t in LAYERS}
    net = O.UNetOracle([(n, ci, co, t, n != "head") for n, ci, co, t in LAYERS], W, B,
                       store_bf16=False)
    x = rng.random((1, 8, 8, 8, 16)).astype(np.float32)
    dd = rng.normal(0, 1, (1, 8, 8, 8, 16))
    net.forward(x)
    g = net.backward(dd)
    eps = 1e-4
    for name, ci, co, t in LAYERS:
        i = (int(rng.integers(co)), int(rng.integers(t)), int(rng.integers(ci)))
        w0 = net.w[name][i]
        net.w[name][i] = w0 + eps
        lp = float((net.forward(x) * dd).sum())
        net.w[name][i] = w0 - eps
        lm = float((net.forward(x) * dd).sum())
        net.w[name][i] = w0
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[name][0][i]) <= 1e-5 * max(1.0, abs(fd)), name


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-39], np.float32)
    r = O.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5


def test_network_size():
    assert 1.4e6 <= n_parameters() <= 1.5e6

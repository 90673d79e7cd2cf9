"""The warm-start MLP's device kernels against the float64 oracle: forward pass, loss and
every parameter gradient (FP32 tolerances), optimiser progress and repeatability."""

import numpy as np
import pytest

from oracle.mlp import forward, loss_and_grad

pytestmark = pytest.mark.gpu

WIDTHS = [2, 64, 64, 64, 4]


def _data(n=512, seed=3):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 2)).astype(np.float32)
    y = np.stack([np.sin(2 * x[:, 0]) + x[:, 1], x[:, 0] * x[:, 1], np.cos(x[:, 1]),
                  x[:, 0] ** 2], axis=1).astype(np.float32)
    return x, y


def test_forward_and_gradients_match_oracle():
    from mdelast_b200.mlp import MLP
    net = MLP(WIDTHS, seed=11)
    x, y = _data()
    p = net.params.astype(np.float64)
    assert np.allclose(net(x), forward(p, WIDTHS, x), rtol=1e-4, atol=1e-5)
    loss, g = net.gradients(x, y)
    lo, go = loss_and_grad(p, WIDTHS, x, y)
    assert abs(loss / lo - 1) < 1e-4
    assert np.max(np.abs(g - go)) / np.max(np.abs(go)) < 2e-4
    # every layer's gradient block, not only the largest entries
    k = 0
    for a, b in zip(WIDTHS[:-1], WIDTHS[1:]):
        blk = slice(k, k + a * b + b)
        k += a * b + b
        assert np.linalg.norm(g[blk] - go[blk]) / np.linalg.norm(go[blk]) < 1e-3


def test_training_reduces_loss_and_repeats_bit_for_bit():
    from mdelast_b200.mlp import MLP
    x, y = _data()
    a, b = MLP(WIDTHS, seed=5), MLP(WIDTHS, seed=5)
    l0, _ = a.gradients(x, y)
    la = a.train(x, y, 1500, lr=2e-3)
    lb = b.train(x, y, 1500, lr=2e-3)
    assert la < 0.02 * l0
    assert la == lb and np.array_equal(a.params, b.params)
    # the loss reported is the oracle's loss of the trained parameters
    lo, _ = loss_and_grad(a.params.astype(np.float64), WIDTHS, x, y)
    assert abs(la / lo - 1) < 1e-3


def test_params_round_trip_and_reset():
    from mdelast_b200.mlp import MLP
    net = MLP(WIDTHS, seed=1)
    p = np.random.default_rng(0).normal(0, 0.1, net.n_params).astype(np.float32)
    net.params = p
    assert np.array_equal(net.params, p)

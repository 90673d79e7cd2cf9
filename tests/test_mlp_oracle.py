"""The warm-start MLP's oracle (float64 numpy) pinned by central finite differences, and the
C-ABI entry points' argument checks without a GPU."""

import numpy as np

from oracle.mlp import forward, loss_and_grad

WIDTHS = [3, 8, 8, 4]


def _setup(seed=0):
    rng = np.random.default_rng(seed)
    n = sum(a * b + b for a, b in zip(WIDTHS[:-1], WIDTHS[1:]))
    return rng.normal(0, 0.5, n), rng.normal(0, 1, (16, 3)), rng.normal(0, 1, (16, 4))


def test_oracle_gradient_matches_finite_differences():
    p, x, y = _setup()
    loss, g = loss_and_grad(p, WIDTHS, x, y)
    h = 1e-6
    fd = np.zeros_like(p)
    for k in range(len(p)):
        e = np.zeros_like(p)
        e[k] = h
        fd[k] = (loss_and_grad(p + e, WIDTHS, x, y)[0] - loss_and_grad(p - e, WIDTHS, x, y)[0]) / (2 * h)
    assert np.max(np.abs(g - fd)) / np.max(np.abs(g)) < 1e-7
    assert loss == np.mean((forward(p, WIDTHS, x) - y) ** 2)


def test_mlp_create_without_device_fails_cleanly():
    import ctypes as C
    import pytest
    from mdelast_b200 import mlp
    try:
        L = mlp.lib()
    except OSError:
        pytest.skip("library not built")
    w = (C.c_int32 * 3)(2, 4, 1)
    h = C.c_void_p()
    assert L.mdelast_mlp_create(0, w, 0, 0, C.byref(h)) == -1  # no layers
    assert L.mdelast_mlp_create(9, w, 0, 0, C.byref(h)) == -1  # too many layers

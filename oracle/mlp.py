"""Test infrastructure (the oracle), not the product: a float64 numpy restatement of the
warm-start MLP (fully connected, exact GELU 0.5 z (1 + erf(z / sqrt 2)) between layers,
linear output, mean-squared-error loss) and of its gradients by the chain rule, used to
check the device's forward and backward kernels. Pinned by central finite differences
(tests/test_mlp_oracle.py). Parameter layout: per layer W (in x out, row-major), then b.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def unpack(params, widths):
    params = np.asarray(params, dtype=np.float64)
    out, k = [], 0
    for a, b in zip(widths[:-1], widths[1:]):
        W = params[k:k + a * b].reshape(a, b)
        k += a * b
        bias = params[k:k + b]
        k += b
        out.append((W, bias))
    assert k == len(params)
    return out


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(params, widths, x):
    layers = unpack(params, widths)
    a = np.asarray(x, dtype=np.float64)
    for l, (W, b) in enumerate(layers):
        z = a @ W + b
        a = gelu(z) if l + 1 < len(layers) else z
    return a


def loss_and_grad(params, widths, x, y):
    """(mean squared error, gradient in the parameter layout)."""
    layers = unpack(params, widths)
    acts, zs = [np.asarray(x, dtype=np.float64)], []
    for l, (W, b) in enumerate(layers):
        z = acts[-1] @ W + b
        zs.append(z)
        acts.append(gelu(z) if l + 1 < len(layers) else z)
    d = acts[-1] - np.asarray(y, dtype=np.float64)
    loss = float(np.mean(d * d))
    dA = 2.0 * d / d.size
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        dZ = dA * gelu_d(zs[l]) if l + 1 < len(layers) else dA
        grads.append((acts[l].T @ dZ, dZ.sum(axis=0)))
        dA = dZ @ W.T
    flat = []
    for dW, db in reversed(grads):
        flat += [dW.ravel(), db]
    return loss, np.concatenate(flat)

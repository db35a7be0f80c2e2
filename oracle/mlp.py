"""CPU oracle of the warm-start network (test infrastructure only).

A float64 numpy restatement of what the FP32 kernels of
``gpu_simulation_b200/csrc/rsv_mlp.cu`` compute: a fully connected network
with GELU (erf form) after every layer but the last, the mean squared error,
and the bias-corrected Adam step (Kingma & Ba, "Adam: A Method for Stochastic
Optimization", 2015, Algorithm 1).  The reference has no learned component, so
there is no reference file to follow; the backward pass here is pinned by
central finite differences in ``tests/test_mlp_oracle.py``.

Weights are packed layer by layer: W_l (widths[l] x widths[l-1], row-major)
then b_l (widths[l]).
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def num_weights(widths) -> int:
    return int(sum(widths[l] * widths[l - 1] + widths[l] for l in range(1, len(widths))))


def unpack(weights, widths):
    """List of (W, b) views of the packed weight vector."""
    out, off = [], 0
    for l in range(1, len(widths)):
        k, n = widths[l - 1], widths[l]
        W = weights[off:off + n * k].reshape(n, k)
        off += n * k
        b = weights[off:off + n]
        off += n
        out.append((W, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(weights, widths, x):
    """(output, cache) for inputs x of shape (batch, widths[0])."""
    weights = np.asarray(weights, dtype=np.float64)
    a = np.asarray(x, dtype=np.float64)
    cache = []
    layers = unpack(weights, widths)
    for i, (W, b) in enumerate(layers):
        z = a @ W.T + b
        cache.append((a, z))
        a = gelu(z) if i + 1 < len(layers) else z
    return a, cache


def backward(weights, widths, cache, dout):
    """Packed gradient of the loss given dLoss/doutput."""
    weights = np.asarray(weights, dtype=np.float64)
    layers = unpack(weights, widths)
    grads = [None] * len(layers)
    dz = np.asarray(dout, dtype=np.float64)
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        a_in, _ = cache[i]
        grads[i] = (dz.T @ a_in, dz.sum(axis=0))
        if i > 0:
            da = dz @ W
            dz = da * gelu_grad(cache[i - 1][1])
    return np.concatenate([np.concatenate([gW.reshape(-1), gb]) for gW, gb in grads])


def mse(out, target):
    """(loss, dLoss/dout) of mean((out - target)^2)."""
    d = np.asarray(out, dtype=np.float64) - np.asarray(target, dtype=np.float64)
    return float(np.mean(d * d)), 2.0 * d / d.size


def adam(p, g, m, v, lr, beta1, beta2, eps, step):
    """One bias-corrected Adam step; returns (p, m, v)."""
    m = beta1 * m + (1.0 - beta1) * g
    v = beta2 * v + (1.0 - beta2) * g * g
    mhat = m / (1.0 - beta1 ** step)
    vhat = v / (1.0 - beta2 ** step)
    return p - lr * mhat / (np.sqrt(vhat) + eps), m, v

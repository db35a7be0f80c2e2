"""Pins of the warm-start network oracle (CPU): its backward pass against
central finite differences, the Adam step against a hand-unrolled case, and
the host-side helpers of gpu_simulation_b200.warmstart (no GPU)."""

from __future__ import annotations

import numpy as np

from oracle import mlp


def small_net(seed=0, widths=(3, 7, 5, 4)):
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(mlp.num_weights(widths)) * 0.5
    x = rng.standard_normal((6, widths[0]))
    t = rng.standard_normal((6, widths[-1]))
    return widths, w, x, t


def loss_of(w, widths, x, t):
    out, _ = mlp.forward(w, widths, x)
    return mlp.mse(out, t)[0]


def test_backward_matches_finite_differences():
    widths, w, x, t = small_net()
    out, cache = mlp.forward(w, widths, x)
    _, dout = mlp.mse(out, t)
    g = mlp.backward(w, widths, cache, dout)
    eps = 1e-6
    fd = np.empty_like(w)
    for i in range(w.size):
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd[i] = (loss_of(wp, widths, x, t) - loss_of(wm, widths, x, t)) / (2 * eps)
    np.testing.assert_allclose(g, fd, atol=1e-8, rtol=1e-6)


def test_gelu_values_and_derivative():
    z = np.linspace(-6, 6, 101)
    # GELU(0) = 0, GELU(z) -> z for large z, -> 0 for very negative z
    assert mlp.gelu(np.array([0.0]))[0] == 0.0
    assert abs(mlp.gelu(np.array([6.0]))[0] - 6.0) < 1e-7
    assert abs(mlp.gelu(np.array([-6.0]))[0]) < 1e-7
    h = 1e-6
    fd = (mlp.gelu(z + h) - mlp.gelu(z - h)) / (2 * h)
    np.testing.assert_allclose(mlp.gelu_grad(z), fd, atol=1e-8)


def test_adam_step_by_hand():
    p, g = np.array([1.0, -2.0]), np.array([0.5, -0.25])
    m = v = np.zeros(2)
    p1, m1, v1 = mlp.adam(p, g, m, v, 0.1, 0.9, 0.999, 1e-8, 1)
    # first step: mhat = g, vhat = g^2 -> p - lr * sign(g) (up to eps)
    np.testing.assert_allclose(p1, p - 0.1 * np.sign(g), atol=1e-7)
    np.testing.assert_allclose(m1, 0.1 * g)
    np.testing.assert_allclose(v1, 0.001 * g * g)


def test_warmstart_host_helpers():
    from gpu_simulation_b200 import warmstart as ws

    x = ws.features([0.2, 1.0, 2.0], 16, 6)
    assert x.shape == (3, 3) and x.dtype == np.float32
    ang = np.array([[0.2, -3.0, 3.1], [0.1, 3.0, -3.1], [0.3, -2.9, 3.0]])
    fields = np.array([1.0, 0.5, 1.5])  # row order is not h order
    lab = ws.unwrap_labels(ang, fields)
    # same angles modulo 2 pi, continuous along increasing h, column means in [-pi, pi]
    np.testing.assert_allclose(np.cos(lab), np.cos(ang), atol=1e-12)
    np.testing.assert_allclose(np.sin(lab), np.sin(ang), atol=1e-12)
    srt = lab[np.argsort(fields)]
    assert np.all(np.abs(np.diff(srt, axis=0)) < 0.5)
    assert np.all(np.abs(lab.mean(axis=0)) <= np.pi)
    hist = np.array([[-1.0, -1.0], [-1.5, -1.9], [-1.999, -1.95], [-2.0, -2.0]])
    steps = ws.steps_to_reach(hist, np.array([-2.0, -2.0]), rel=1e-3)
    assert list(steps) == [2, 3]
    never = ws.steps_to_reach(hist, np.array([-3.0, -2.0]), rel=1e-3)
    assert never[0] == -1
    w = ws.init_weights((3, 256, 256, 192), seed=1)
    assert w.size == mlp.num_weights((3, 256, 256, 192)) and w.dtype == np.float32

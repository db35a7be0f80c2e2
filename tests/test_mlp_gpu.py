"""Warm-start network kernels against the CPU oracle (oracle/mlp.py), the
fused Adam steps, and the gain of the trained warm start over random init."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import mlp

pytestmark = pytest.mark.gpu

WIDTHS = (3, 256, 256, 192)


def setup(batch=96, seed=0, widths=WIDTHS):
    import torch

    from gpu_simulation_b200.warmstart import WarmStartMLP

    net = WarmStartMLP(widths, seed=seed)
    rng = np.random.default_rng(seed + 1)
    x = rng.uniform(-1.0, 2.0, (batch, widths[0])).astype(np.float32)
    t = rng.uniform(-3.0, 3.0, (batch, widths[-1])).astype(np.float32)
    return net, x, t, torch


def test_forward_matches_oracle():
    net, x, _, torch = setup()
    out = net.forward(torch.from_numpy(x)).cpu().numpy()
    ref, _ = mlp.forward(net.weights.cpu().numpy().astype(np.float64), WIDTHS, x.astype(np.float64))
    # FP32 with FP32 accumulation over K <= 256
    np.testing.assert_allclose(out, ref, atol=2e-5 * np.abs(ref).max(), rtol=1e-4)


def test_backward_matches_oracle():
    net, x, t, torch = setup()
    loss, grad = net.gradient(torch.from_numpy(x), torch.from_numpy(t))
    w64 = net.weights.cpu().numpy().astype(np.float64)
    out, cache = mlp.forward(w64, WIDTHS, x.astype(np.float64))
    l_ref, dout = mlp.mse(out, t.astype(np.float64))
    g_ref = mlp.backward(w64, WIDTHS, cache, dout)
    assert abs(loss.item() - l_ref) < 1e-5 * abs(l_ref)
    g = grad.cpu().numpy()
    np.testing.assert_allclose(g, g_ref, atol=1e-5 * np.abs(g_ref).max(), rtol=1e-3)


def test_backward_other_shapes():
    # ragged sizes (not multiples of the 64-wide tiles), one and two layers
    for widths, batch in (((5, 33, 7), 13), ((2, 9), 1), ((3, 70, 65, 130), 200)):
        net, x, t, torch = setup(batch=batch, seed=3, widths=widths)
        _, grad = net.gradient(torch.from_numpy(x), torch.from_numpy(t))
        w64 = net.weights.cpu().numpy().astype(np.float64)
        out, cache = mlp.forward(w64, widths, x.astype(np.float64))
        _, dout = mlp.mse(out, t.astype(np.float64))
        g_ref = mlp.backward(w64, widths, cache, dout)
        np.testing.assert_allclose(grad.cpu().numpy(), g_ref, atol=1e-5 * np.abs(g_ref).max(), rtol=1e-3)


def test_adam_kernels_match_oracle():
    import torch

    from gpu_simulation_b200._lib import check, load_library

    lib = load_library()
    rng = np.random.default_rng(4)
    for dtype, fn, tol in ((torch.float64, lib.rsv_adam_f64, 1e-14), (torch.float32, lib.rsv_adam_f32, 1e-6)):
        p0 = rng.standard_normal(1000)
        p = torch.tensor(p0, dtype=dtype, device="cuda")
        m = torch.zeros_like(p)
        v = torch.zeros_like(p)
        pr, mr, vr = p0.copy(), np.zeros(1000), np.zeros(1000)
        for step in range(1, 6):
            g0 = rng.standard_normal(1000)
            g = torch.tensor(g0, dtype=dtype, device="cuda")
            check(fn(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), 1000, 0.05, 0.9, 0.999, 1e-8, step,
                     torch.cuda.current_stream().cuda_stream))
            g_used = g.cpu().numpy().astype(np.float64)
            pr, mr, vr = mlp.adam(pr, g_used, mr, vr, 0.05, 0.9, 0.999, 1e-8, step)
        np.testing.assert_allclose(p.cpu().numpy(), pr, atol=tol * 10, rtol=tol * 10)


def test_training_reduces_loss():
    net, x, t, torch = setup(batch=128, widths=(3, 64, 64, 8))
    # a smooth target of the inputs
    y = np.stack([np.sin(x[:, 0] * (k + 1)) + 0.3 * x[:, 1] for k in range(8)], axis=1).astype(np.float32)
    losses = net.train(torch.from_numpy(x), torch.from_numpy(y), steps=400, lr=3e-3)
    assert losses[-1] < 0.05 * losses[0]


def test_warm_start_gains_over_random_init():
    from gpu_simulation_b200.warmstart import warm_start_experiment

    r = warm_start_experiment(num_qubits=8, num_layers=3, train_count=96, test_count=24, vqe_steps=150,
                              mlp_schedule=((1000, 3e-3), (1000, 1e-3)))
    assert r["warm_reached_fraction"] >= 0.9
    assert r["warm_steps_median"] < r["plain_steps_median"]
    assert r["warm_initial_gap_median"] < r["plain_initial_gap_median"]

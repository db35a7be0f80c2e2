"""The two backward schedules (uncompute: three buffers, psi un-computed with
lambda; checkpoint: psi read from forward checkpoints, only lambda written)
against the oracle at 1e-10 and against each other."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("n,L,h", [
    (13, 1, 0.8), (13, 3, 1.1), (14, 2, 1.0), (15, 5, 0.4), (16, 4, 1.3), (17, 3, 0.9),
    (19, 2, 1.0), (20, 3, 0.6), (21, 2, 0.8), (22, 2, 1.7),
])
def test_both_schedules_match_oracle(n, L, h):
    p = np.random.default_rng(500 + 7 * n + L).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    eng = Engine(n, L, h)
    out = {}
    for mode in ("uncompute", "checkpoint"):
        eng.set_backward_mode(mode)
        info = eng.backward_mode()
        assert info["checkpoint"] == (mode == "checkpoint")
        e, g = eng.energy_and_grad(p)
        assert abs(e - e_ref) < TOL, (mode, e, e_ref)
        np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0, err_msg=mode)
        out[mode] = (e, g)
    assert abs(out["uncompute"][0] - out["checkpoint"][0]) < 1e-12
    np.testing.assert_allclose(out["uncompute"][1], out["checkpoint"][1], atol=1e-12, rtol=0)


def test_auto_mode_and_buffers():
    eng = Engine(14, 3, 1.0)
    eng.set_analytic_layers(0)  # every layer on tile passes
    info = eng.backward_mode()
    assert info["mode"] == "auto" and info["checkpoint"] and info["state_buffers"] == 2 * 2 + 1
    eng.set_backward_mode("uncompute")
    assert eng.backward_mode()["state_buffers"] == 3
    # layers 0..2 as a matrix-product state: only chi and lambda remain
    eng.set_analytic_layers(3)
    assert eng.backward_mode()["state_buffers"] == 2
    eng.set_backward_mode("auto")
    assert eng.backward_mode()["checkpoint"] and eng.backward_mode()["state_buffers"] == 2
    assert Engine(12, 3, 1.0).backward_mode()["checkpoint"] is False  # one tile: in place


def test_checkpoint_device_split_forward_backward():
    # the autograd split keeps the checkpoints between forward and backward
    import torch

    n, L, h = 16, 3, 0.9
    p = np.random.default_rng(3).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    from gpu_simulation_b200 import ring_ising_energy

    eng = Engine(n, L, h)
    x = torch.tensor(p, device="cuda", requires_grad=True)
    e = ring_ising_energy(x, eng)
    e.backward()
    assert abs(e.item() - e_ref) < TOL
    np.testing.assert_allclose(x.grad.cpu().numpy(), g_ref, atol=TOL, rtol=0)


def test_largest_single_gpu_circuit_takes_the_checkpoint_schedule():
    """n = 31, L = 4: the checkpoint schedule's four state buffers (128 GiB, as
    many bytes as the reference's four buffers) are the automatic choice and
    agree with the two-buffer uncompute schedule."""
    import torch

    torch.cuda.empty_cache()
    n, L, h = 31, 4, 1.0
    p = np.random.default_rng(31).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    eng = Engine(n, L, h)
    try:
        info = eng.backward_mode()
        assert info["mode"] == "auto" and info["checkpoint"] and info["state_buffers"] == 4, info
        e_ck, g_ck = eng.energy_and_grad(p)
        eng.set_backward_mode("uncompute")
        e_un, g_un = eng.energy_and_grad(p)
    finally:
        eng.close()
    assert abs(e_ck - e_un) < 1e-12
    np.testing.assert_allclose(g_ck, g_un, atol=1e-12, rtol=0)

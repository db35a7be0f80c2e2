"""Device-resident training loop (the reference's standalone workflow): the
reference's published known answers (20 plain gradient-descent steps,
stepsize 0.08, seed 7, init 0.3 N(0,1), h=1, L=2), CUDA-graph replay equal to
plain launches, and the per-step metrics equal to a host-side loop."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from gpu_simulation_b200 import Engine
from gpu_simulation_b200.training import make_initial_params, run_gradient_descent_device, run_standalone

pytestmark = pytest.mark.gpu

DATA = json.loads((Path(__file__).parent / "golden" / "csv_known_answers.json").read_text())


@pytest.mark.parametrize("n", [8, 12, 16, 20])
def test_device_loop_reproduces_reference_final_energy(n):
    proto = DATA["protocol"]
    r = run_standalone(n, proto["layers"], proto["steps"], proto["stepsize"], field=proto["field"],
                       seed=proto["seed"], init_scale=proto["init_scale"])
    for method, value in DATA["final_energy"][str(n)].items():
        assert abs(r.final_energy - value) < 1e-9, (n, method, r.final_energy, value)
    assert len(r.step_metrics) == proto["steps"]


def test_graph_replay_equals_launches_and_host_loop():
    n, L, steps, lr = 14, 3, 12, 0.05
    p0 = make_initial_params(n, L, 11, 0.3)
    eng = Engine(n, L, 0.8)
    rg = run_gradient_descent_device(eng, p0, steps, lr, use_graph=True)
    rl = run_gradient_descent_device(eng, p0, steps, lr, use_graph=False)
    assert np.array_equal(rg.final_params, rl.final_params)
    assert [m.energy for m in rg.step_metrics] == [m.energy for m in rl.step_metrics]
    # host loop with the same update
    p = p0.copy()
    energies = []
    for _ in range(steps):
        e, g = eng.energy_and_grad(p)
        energies.append(e)
        p = p - lr * g.reshape(p.shape)
    np.testing.assert_allclose(rg.final_params, p, atol=1e-12, rtol=0)
    np.testing.assert_allclose([m.energy for m in rg.step_metrics], energies, atol=1e-12, rtol=0)
    assert all(m.grad_norm > 0 for m in rg.step_metrics)


@pytest.mark.parametrize("n,L,use_graph", [(12, 3, True), (12, 3, False), (14, 2, True)])
def test_device_adam_matches_torch_adam(n, L, use_graph):
    # the fused device Adam loop follows torch.optim.Adam over the autograd Function
    import torch

    from gpu_simulation_b200 import ring_ising_energy
    from gpu_simulation_b200.training import run_adam_device

    steps, lr = 20, 0.05
    p0 = np.random.default_rng(7).uniform(0.0, 2.0 * np.pi, (L, n, 2))
    eng = Engine(n, L, 1.0)
    x = torch.tensor(p0, device="cuda", requires_grad=True)
    opt = torch.optim.Adam([x], lr=lr)
    energies = []
    for _ in range(steps):
        opt.zero_grad()
        e = ring_ising_energy(x, eng)
        e.backward()
        opt.step()
        energies.append(float(e.item()))
    out = run_adam_device(eng, p0, steps, lr=lr, use_graph=use_graph)
    np.testing.assert_allclose(out["energies"], energies, atol=1e-9, rtol=0)
    np.testing.assert_allclose(out["params"], x.detach().cpu().numpy().reshape(-1), atol=1e-9, rtol=0)
    assert out["energies"][-1] < out["energies"][0]

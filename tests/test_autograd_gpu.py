"""torch.autograd.Function around the energy: backward = the adjoint kernels."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu


def test_backward_matches_oracle_small():
    import torch
    from gpu_simulation_b200 import ring_ising_energy

    n, L, h = 8, 3, 1.0
    p0 = np.random.default_rng(3).uniform(0, 2 * np.pi, (L, n, 2))
    eng = Engine(n, L, h)
    p = torch.tensor(p0, device="cuda", requires_grad=True)
    e = ring_ising_energy(p, eng)
    e.backward()
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p0.reshape(-1))
    assert abs(e.item() - e_ref) < 1e-10
    np.testing.assert_allclose(p.grad.cpu().numpy().reshape(-1), g_ref, atol=1e-10, rtol=0)


def test_finite_differences_and_reference_gradient_at_20x8():
    """Differentiation check config: n=20, L=8, seed 7 angles U[0, 2pi);
    64 parameters vs central differences (step 1e-5, tol 1e-7) and all
    parameters vs the oracle gradient (tol 1e-10)."""
    import torch
    from gpu_simulation_b200 import ring_ising_energy

    n, L, h, seed = 20, 8, 1.0, 7
    p0 = np.random.default_rng(seed).uniform(0, 2 * np.pi, 2 * n * L)
    eng = Engine(n, L, h)
    p = torch.tensor(p0, device="cuda", requires_grad=True)
    ring_ising_energy(p, eng).backward()
    g = p.grad.cpu().numpy()
    _, g_ref = oracle.energy_and_grad(n, L, h, p0)
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)
    idx = np.random.default_rng(seed + 1).choice(p0.size, 64, replace=False)
    step = 1e-5
    for k in idx:
        pp, pm = p0.copy(), p0.copy()
        pp[k] += step
        pm[k] -= step
        fd = (eng.energy(pp) - eng.energy(pm)) / (2 * step)
        assert abs(fd - g[k]) < 1e-7, (k, fd, g[k])


def test_second_forward_before_backward_recomputes():
    import torch
    from gpu_simulation_b200 import ring_ising_energy

    n, L, h = 10, 2, 0.8
    eng = Engine(n, L, h)
    a0 = np.random.default_rng(1).uniform(0, 2 * np.pi, 2 * n * L)
    b0 = np.random.default_rng(2).uniform(0, 2 * np.pi, 2 * n * L)
    a = torch.tensor(a0, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    ea = ring_ising_energy(a, eng)
    eb = ring_ising_energy(b, eng)
    (ea + 2.0 * eb).backward()
    _, ga = oracle.energy_and_grad(n, L, h, a0)
    _, gb = oracle.energy_and_grad(n, L, h, b0)
    np.testing.assert_allclose(a.grad.cpu().numpy(), ga, atol=1e-10, rtol=0)
    np.testing.assert_allclose(b.grad.cpu().numpy(), 2.0 * gb, atol=1e-10, rtol=0)


def test_adam_steps_through_the_function_lower_the_energy():
    import torch
    from gpu_simulation_b200 import ring_ising_energy

    n, L, h = 20, 8, 1.0
    eng = Engine(n, L, h)
    p = torch.tensor(np.random.default_rng(7).uniform(0, 2 * np.pi, (L, n, 2)), device="cuda",
                     requires_grad=True)
    opt = torch.optim.Adam([p], lr=0.05)
    energies = []
    for _ in range(100):
        opt.zero_grad()
        e = ring_ising_energy(p, eng)
        e.backward()
        opt.step()
        energies.append(e.item())
    assert energies[-1] < energies[0] - 1.0
    assert energies[-1] >= oracle.ground_energy_free_fermion(n, h) - 1e-9

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


def test_backward_status_stale_state_recomputes_and_other_failures_raise():
    import ctypes

    import torch
    from gpu_simulation_b200 import _lib, ring_ising_energy

    n, L, h = 8, 2, 0.9
    eng = Engine(n, L, h)
    a = torch.tensor(np.random.default_rng(4).uniform(0, 2 * np.pi, 2 * n * L), device="cuda")
    e = torch.empty(1, dtype=torch.float64, device="cuda")
    g = torch.empty_like(a)
    ga, gb = ctypes.c_ulonglong(), ctypes.c_ulonglong()
    lib = eng._lib
    _lib.check(lib.rsv_forward_device(eng._h, a.data_ptr(), a.numel(), e.data_ptr(), ctypes.byref(ga), None))
    _lib.check(lib.rsv_forward_device(eng._h, a.data_ptr(), a.numel(), e.data_ptr(), ctypes.byref(gb), None))
    # the first forward's state is gone: a dedicated status, not a bad argument
    assert lib.rsv_backward_device(eng._h, ga.value, g.data_ptr(), None) == _lib.RSV_ERR_STALE_STATE
    assert lib.rsv_backward_device(eng._h, gb.value, None, None) == _lib.RSV_ERR_INVALID_ARGUMENT
    _lib.check(lib.rsv_backward_device(eng._h, gb.value, g.data_ptr(), None))

    class FailingLib:
        """The engine's library with a backward that reports a CUDA error."""

        def __getattr__(self, name):
            if name == "rsv_backward_device":
                return lambda *args: 2  # RSV_ERR_CUDA
            return getattr(lib, name)

    eng._lib = FailingLib()
    p = a.clone().requires_grad_(True)
    with pytest.raises(RuntimeError):
        ring_ising_energy(p, eng).backward()
    eng._lib = lib

"""Gate-level inverse walk (gradient_strategy "inverse_walk_cuQuantum"): RY, RZ
and CNOT as separate kernels and the adjoint walk, a second GPU path checked
against the oracle's gate-level mode and against the structured engine."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("n,L,h", [(2, 1, 0.7), (2, 3, 1.0), (3, 2, 1.1), (5, 3, 0.4), (8, 2, 1.0),
                                   (11, 2, 1.3), (12, 3, 1.0), (13, 2, 0.8), (16, 2, 1.2), (20, 2, 1.0)])
def test_gate_level_matches_oracle_and_structured(n, L, h):
    p = np.random.default_rng(900 + 13 * n + L).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p, mode="inverse_walk")
    gate = Engine(n, L, h, gradient_strategy="inverse_walk_cuQuantum")
    e, g = gate.energy_and_grad(p)
    assert abs(e - e_ref) < TOL, (e, e_ref)
    np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0)
    e_s, g_s = Engine(n, L, h).energy_and_grad(p)
    assert abs(e - e_s) < 1e-11
    np.testing.assert_allclose(g, g_s, atol=1e-11, rtol=0)
    assert gate.energy(p) == pytest.approx(e, abs=1e-13)


def test_gate_level_profile_and_device_entry():
    import torch

    n, L, h = 10, 3, 0.9
    p = np.random.default_rng(1).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    eng = Engine(n, L, h, gradient_strategy="inverse_walk_cuquantum")
    e, g = eng.energy_and_grad(p)
    prof = eng.profile_energy_and_grad(p)
    assert prof["energy"] == pytest.approx(e, abs=1e-13)
    np.testing.assert_allclose(prof["gradient"], g, atol=1e-13, rtol=0)
    dp = torch.tensor(p, device="cuda")
    de = torch.empty(1, dtype=torch.float64, device="cuda")
    dg = torch.empty_like(dp)
    eng.energy_and_grad_device(dp, de, dg)
    torch.cuda.synchronize()
    assert abs(de.item() - e) < 1e-12
    np.testing.assert_allclose(dg.cpu().numpy(), g, atol=1e-12, rtol=0)

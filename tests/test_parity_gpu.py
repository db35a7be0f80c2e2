"""Parity of the CUDA engine (through the C ABI) with the CPU oracle, at sizes
the oracle finishes in seconds, plus size-independent properties."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-10  # absolute, energy and gradient

CASES = [
    (2, 1, 0.7), (2, 2, 1.0), (3, 1, 1.0), (3, 3, 1.1), (4, 2, 1.0), (5, 4, 0.3), (6, 2, 1.1),
    (7, 5, 0.9), (8, 3, 1.0), (9, 2, 2.0), (10, 3, 0.5), (11, 2, 1.3), (12, 1, 1.0),
    (12, 3, 1.0), (13, 1, 0.8), (13, 2, 0.8), (14, 3, 1.0), (15, 2, 0.6), (16, 2, 1.2),
    (17, 3, 1.0), (18, 2, 1.4), (19, 2, 1.0), (20, 3, 1.0), (21, 2, 0.9), (22, 2, 1.0),
]


def params_for(n, L, seed):
    return np.random.default_rng(seed).uniform(0.0, 2.0 * np.pi, 2 * n * L)


@pytest.mark.parametrize("n,L,h", CASES)
def test_energy_and_gradient_match_oracle(n, L, h):
    p = params_for(n, L, 1000 + 31 * n + L)
    eng = Engine(n, L, h)
    e, g = eng.energy_and_grad(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert abs(e - e_ref) < TOL, (e, e_ref)
    np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0)
    e_only = eng.energy(p)
    assert abs(e_only - e) < 1e-13


@pytest.mark.parametrize("n,L", [(8, 2), (14, 3), (20, 2)])
def test_small_init_scale_like_reference_tests(n, L):
    # the reference's own tests use 0.2 * N(0,1) parameters
    p = 0.2 * np.random.default_rng(123).standard_normal(2 * n * L)
    e, g = Engine(n, L, 1.0).energy_and_grad(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, 1.0, p)
    assert abs(e - e_ref) < TOL
    np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0)


def test_results_are_deterministic():
    n, L = 20, 4
    p = params_for(n, L, 5)
    eng = Engine(n, L, 1.0)
    e1, g1 = eng.energy_and_grad(p)
    e2, g2 = eng.energy_and_grad(p)
    assert e1 == e2
    assert np.array_equal(g1, g2)


def test_device_entry_point_matches_host_entry_point():
    import torch

    n, L = 16, 3
    p = params_for(n, L, 9)
    eng = Engine(n, L, 0.8)
    e, g = eng.energy_and_grad(p)
    dp = torch.tensor(p, device="cuda")
    de = torch.empty(1, dtype=torch.float64, device="cuda")
    dg = torch.empty_like(dp)
    eng.energy_and_grad_device(dp, de, dg)
    torch.cuda.synchronize()
    assert abs(de.item() - e) < 1e-12
    np.testing.assert_allclose(dg.cpu().numpy(), g, atol=1e-12, rtol=0)


@pytest.mark.parametrize("n,L", [(20, 4), (24, 2)])
def test_energy_is_affine_in_the_field(n, L):
    # the state does not depend on h, so E(h) and dE/dp are affine in h
    p = params_for(n, L, 17)
    hs = (0.3, 1.0, 1.7)
    res = [Engine(n, L, h).energy_and_grad(p) for h in hs]
    w = (hs[2] - hs[1]) / (hs[2] - hs[0])
    e_mid = w * res[0][0] + (1 - w) * res[2][0]
    g_mid = w * res[0][1] + (1 - w) * res[2][1]
    assert abs(res[1][0] - e_mid) < 1e-9
    np.testing.assert_allclose(res[1][1], g_mid, atol=1e-9, rtol=0)


def test_zero_rotation_angles_give_the_classical_ferromagnet():
    # theta = 0 keeps |0...0>: E = -n exactly and all phi gradients vanish
    n, L = 24, 3
    p = np.zeros((L, n, 2))
    p[..., 1] = np.random.default_rng(3).uniform(0, 2 * np.pi, (L, n))
    e, g = Engine(n, L, 1.0).energy_and_grad(p.reshape(-1))
    assert abs(e + n) < 1e-12
    assert np.max(np.abs(g.reshape(L, n, 2)[..., 1])) < 1e-12


def test_gradient_matches_central_differences_at_24_qubits():
    n, L, h = 24, 4, 1.0
    p = params_for(n, L, 7)
    eng = Engine(n, L, h)
    _, g = eng.energy_and_grad(p)
    step = 1e-5
    for k in np.random.default_rng(8).choice(p.size, 6, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[k] += step
        pm[k] -= step
        fd = (eng.energy(pp) - eng.energy(pm)) / (2 * step)
        assert abs(fd - g[k]) < 1e-6, (k, fd, g[k])


def test_wrong_parameter_count_raises_value_error():
    eng = Engine(6, 2, 1.0)
    with pytest.raises(ValueError):
        eng.energy_and_grad(np.zeros(5))


def test_engine_matches_reference_golden_vectors():
    """All golden vectors of the reference's own extension (including n=20)."""
    import json
    from pathlib import Path

    data = json.loads((Path(__file__).parent / "golden" / "ref_golden.json").read_text())
    for case in data["cases"]:
        n, L, h = case["n"], case["L"], case["h"]
        p = np.random.default_rng(case["seed"]).uniform(0.0, 2.0 * np.pi, 2 * n * L)
        e, g = Engine(n, L, h).energy_and_grad(p)
        assert abs(e - case["energy"]) < TOL, (n, L)
        np.testing.assert_allclose(g, np.asarray(case["gradient"]), atol=TOL, rtol=0)

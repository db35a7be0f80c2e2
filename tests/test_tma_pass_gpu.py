"""Backward passes on the TMA-fed kernel (rsv_pass_tma.cu).

The kernel takes the 11-bit backward passes of the checkpoint schedule whose
psi and lambda are read in natural order; every other pass keeps its cp.async
kernel, so a circuit can mix both within one call (and within one layer's
gradient correction, which follows each kernel's rotation order).  Results
must agree with the all-cp.async engine to rounding and with the oracle or
the reference rebuild (oracle/_ref) at 1e-10.
"""

from __future__ import annotations

import gc

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine
from tests.refmod import load_reference_module

pytestmark = pytest.mark.gpu

ref = load_reference_module()


def _both_kernels(n, L, h, p):
    eng = Engine(n, L, h)
    try:
        k = eng.kernels()
        assert k["tma"] and k["tma_passes"] > 0, k
        e1, g1 = eng.energy_and_grad(p)
        e1b, g1b = eng.energy_and_grad(p)
        eng.set_kernels(tma=False)
        assert eng.kernels()["tma_passes"] == 0
        e0, g0 = eng.energy_and_grad(p)
        eng.set_kernels(tma=True)
        e2, g2 = eng.energy_and_grad(p)
    finally:
        eng.close()
    assert e1 == e1b and np.array_equal(g1, g1b)  # deterministic
    assert e2 == e1 and np.array_equal(g2, g1)    # re-planned maps, same result
    assert abs(e1 - e0) < 1e-12
    np.testing.assert_allclose(g1, g0, atol=1e-12, rtol=0)
    return e1, g1


@pytest.mark.parametrize("n,L,h", [(23, 4, 0.9), (24, 4, 1.0), (24, 6, 1.3)])
def test_tma_passes_match_oracle(n, L, h):
    p = np.random.default_rng(700 + n + L).uniform(0, 2 * np.pi, 2 * n * L)
    e, g = _both_kernels(n, L, h, p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert abs(e - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


@pytest.mark.skipif(ref is None, reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("n,L,h", [(26, 5, 0.7), (27, 4, 1.0), (28, 5, 1.1), (29, 4, 0.8)])
def test_tma_passes_match_reference(n, L, h):
    p = np.random.default_rng(900 + n + L).uniform(0, 2 * np.pi, 2 * n * L)
    rb = ref.RingIsingCudaBackend(n, L, h, "structured_adjoint", 8, False)
    r = rb.energy_and_grad(p, True, False)
    e_ref, g_ref = float(r["energy"]), np.array(r["gradient"])
    del rb, r
    gc.collect()
    e, g = _both_kernels(n, L, h, p)
    assert abs(e - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


@pytest.mark.parametrize("n,L,h", [(23, 4, 0.8), (24, 4, 1.0), (28, 4, 1.0)])
def test_fused_energy_matches_separate_energy(n, L, h):
    """The last layer's first backward pass applies the field terms on its tile,
    and at n=28 the middle pass those of its own wires (default): energy and
    gradient equal the separate energy kernels' to rounding; energy-only calls
    and the forward/backward device split keep the whole energy kernel (the
    middle pass still takes its wires' phi sums) and agree too."""
    import torch

    from gpu_simulation_b200 import ring_ising_energy

    p = np.random.default_rng(1300 + n + L).uniform(0, 2 * np.pi, 2 * n * L)
    eng = Engine(n, L, h)
    try:
        k = eng.kernels()
        assert k["tma"] and k["fused_energy"], k
        desc = eng.describe().splitlines()[0]
        assert "fused_energy: backward pass 0 applies" in desc
        if n == 28:  # the middle pass (wires 12..19) takes the terms of its wires too
            assert "backward pass 1 applies 7" in desc, desc
        e1, g1 = eng.energy_and_grad(p)
        e1b, g1b = eng.energy_and_grad(p)
        e_only = eng.energy(p)
        t = torch.tensor(p, device="cuda", requires_grad=True)
        e_ad = ring_ising_energy(t, eng)
        e_ad.backward()
        g_ad = t.grad.cpu().numpy()
        eng.set_kernels(tma=True, fused_energy=False)
        assert "fused_energy" not in eng.describe().splitlines()[0]
        e0, g0 = eng.energy_and_grad(p)
    finally:
        eng.close()
    assert e1 == e1b and np.array_equal(g1, g1b)
    assert abs(e1 - e0) < 1e-12 and abs(e_only - e0) < 1e-12 and abs(float(e_ad) - e0) < 1e-12
    np.testing.assert_allclose(g1, g0, atol=1e-12, rtol=0)
    np.testing.assert_allclose(g_ad, g0, atol=1e-12, rtol=0)


def test_fused_energy_follows_set_field():
    """The fused field terms and their phase table take the backend's current
    field, not the one it was planned with."""
    n, L = 28, 4
    p = np.random.default_rng(1400).uniform(0, 2 * np.pi, 2 * n * L)
    eng = Engine(n, L, 1.0)
    try:
        eng.set_field(0.55)
        e1, g1 = eng.energy_and_grad(p)
    finally:
        eng.close()
    fresh = Engine(n, L, 0.55)
    try:
        e0, g0 = fresh.energy_and_grad(p)
    finally:
        fresh.close()
    assert abs(e1 - e0) < 1e-12
    np.testing.assert_allclose(g1, g0, atol=1e-12, rtol=0)

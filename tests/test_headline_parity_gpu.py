"""Parity at the measured configurations, against the reference's own
structured_adjoint extension rebuilt for sm_100a (oracle/_ref) on the same GPU:

* one energy_and_grad at n=28, L=4 and n=30, L=4 (h = J = 1, seed-7 angles
  U[0, 2pi)), the large single-circuit workload the benchmark times;
* the autograd Function at n=20, L=8 (the differentiation check), whose
  backward must equal the reference gradient.

Energy and every gradient entry agree to 1e-10 absolute.  The reference runs
first and is freed before the engine allocates (at n=30 each needs 64 GiB).
"""

from __future__ import annotations

import gc

import numpy as np
import pytest

from gpu_simulation_b200 import Engine
from tests.refmod import load_reference_module

pytestmark = pytest.mark.gpu

ref = load_reference_module()
needs_ref = pytest.mark.skipif(ref is None, reason="oracle/_ref not built (make -C oracle ref)")

TOL = 1e-10


def _reference(n, L, h, p):
    rb = ref.RingIsingCudaBackend(n, L, h, "structured_adjoint", 8, False)
    r = rb.energy_and_grad(p, True, False)
    e, g = float(r["energy"]), np.array(r["gradient"], dtype=np.float64)
    del rb, r
    gc.collect()
    return e, g


@needs_ref
@pytest.mark.parametrize("n", [28, 30])
def test_large_single_circuit_matches_reference(n):
    L, h = 4, 1.0
    p = np.random.default_rng(7).uniform(0, 2 * np.pi, 2 * n * L)
    e_ref, g_ref = _reference(n, L, h, p)
    eng = Engine(n, L, h)
    try:
        e, g = eng.energy_and_grad(p)
        # the host and the device entry points run the same kernels
        e2, g2 = eng.energy_and_grad(p)
    finally:
        eng.close()
    assert abs(e - e_ref) < TOL, (n, e, e_ref)
    np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0)
    assert e2 == e and np.array_equal(g2, g)  # deterministic reductions


@needs_ref
def test_autograd_at_20x8_matches_reference_gradient():
    import torch
    from gpu_simulation_b200 import ring_ising_energy

    n, L, h = 20, 8, 1.0
    p0 = np.random.default_rng(7).uniform(0, 2 * np.pi, 2 * n * L)
    e_ref, g_ref = _reference(n, L, h, p0)
    eng = Engine(n, L, h)
    try:
        p = torch.tensor(p0.reshape(L, n, 2), device="cuda", requires_grad=True)
        e = ring_ising_energy(p, eng)
        e.backward()
        g = p.grad.detach().cpu().numpy().reshape(-1)
    finally:
        eng.close()
    assert abs(e.item() - e_ref) < TOL
    np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0)

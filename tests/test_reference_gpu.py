"""Engine vs the reference's own structured_adjoint extension rebuilt for
sm_100a (oracle/_ref), on the same GPU, at 1e-10 absolute."""

from __future__ import annotations

import numpy as np
import pytest

from gpu_simulation_b200 import Engine
from tests.refmod import load_reference_module

pytestmark = pytest.mark.gpu

ref = load_reference_module()
needs_ref = pytest.mark.skipif(ref is None, reason="oracle/_ref not built (make -C oracle ref)")


@needs_ref
@pytest.mark.parametrize("n,L,h", [
    (2, 2, 0.7), (4, 2, 1.0), (6, 3, 1.1), (8, 4, 1.0), (10, 2, 0.9), (12, 3, 1.0),
    (15, 2, 1.0), (16, 4, 0.7), (19, 2, 1.0), (20, 4, 1.0), (22, 2, 1.3), (24, 2, 1.0),
])
def test_engine_matches_reference_structured_adjoint(n, L, h):
    p = np.random.default_rng(50 + n + L).uniform(0, 2 * np.pi, 2 * n * L)
    r = ref.RingIsingCudaBackend(n, L, h, "structured_adjoint", 8, False).energy_and_grad(p, True, False)
    e, g = Engine(n, L, h).energy_and_grad(p)
    assert abs(e - r["energy"]) < 1e-10
    np.testing.assert_allclose(g, np.asarray(r["gradient"]), atol=1e-10, rtol=0)


@needs_ref
@pytest.mark.parametrize("width", [1, 2, 4, 8])
def test_engine_matches_every_reference_chunk_width(width):
    n, L, h = 10, 2, 0.9
    p = np.random.default_rng(2030).uniform(0, 2 * np.pi, 2 * n * L)
    r = ref.RingIsingCudaBackend(n, L, h, "structured_adjoint", width, False).energy_and_grad(p, True, False)
    e, g = Engine(n, L, h).energy_and_grad(p)
    assert abs(e - r["energy"]) < 1e-10
    np.testing.assert_allclose(g, np.asarray(r["gradient"]), atol=1e-10, rtol=0)

"""Every setting of the analytic leading layers (0: all tile passes, 1: layer-0
backward from one read of lambda, 2 and 3: the first layers as a matrix-product
state of bond 2 or 4) against the oracle at 1e-10, in both backward schedules,
and against each other."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("n,L,h", [
    (13, 2, 0.9), (14, 3, 1.1), (15, 4, 0.6), (16, 3, 1.4), (17, 5, 0.8), (20, 4, 1.0), (21, 3, 1.3),
])
def test_every_setting_matches_oracle(n, L, h):
    p = np.random.default_rng(900 + 3 * n + L).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    eng = Engine(n, L, h)
    results = {}
    for k in (0, 1, 2, 3):
        eng.set_analytic_layers(k)
        info = eng.analytic_layers()
        assert info["max_layers"] == k
        assert info["used"] == (min(L, k) if k >= 2 else k)
        for mode in ("uncompute", "checkpoint"):
            eng.set_backward_mode(mode)
            e, g = eng.energy_and_grad(p)
            assert abs(e - e_ref) < TOL, (k, mode, e, e_ref)
            np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0, err_msg=f"analytic={k} {mode}")
            results[(k, mode)] = g
    base = results[(0, "checkpoint")]
    for key, g in results.items():
        np.testing.assert_allclose(g, base, atol=1e-12, rtol=0, err_msg=str(key))


def test_rejects_out_of_range_setting():
    eng = Engine(13, 2, 1.0)
    with pytest.raises(ValueError):
        eng.set_analytic_layers(4)
    with pytest.raises(ValueError):
        eng.set_analytic_layers(-1)
    assert eng.analytic_layers()["max_layers"] == 3

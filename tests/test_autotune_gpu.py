"""The autotuner (rsv_autotune): it times the plan candidates, every one of
which must compute the same energy and gradient, keeps the fastest, caches
the choice per device and shape, and the chosen plan matches the oracle."""

from __future__ import annotations

import re

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,L,h", [(14, 4, 0.9), (20, 3, 1.1), (24, 4, 1.0)])
def test_autotune_candidates_agree_and_choice_matches_oracle(n, L, h):
    p = np.random.default_rng(400 + n + L).uniform(0, 2 * np.pi, 2 * n * L)
    eng = Engine(n, L, h)
    report = eng.autotune(p, repeats=2, force=True)
    cands = re.findall(r"^candidate .*: ([0-9.eE+-]+) ms$", report, re.M)
    assert len(cands) >= 2, report
    chosen = float(re.search(r"^chosen .*: ([0-9.eE+-]+) ms$", report, re.M).group(1))
    assert chosen == min(float(c) for c in cands)
    spread = float(re.search(r"between candidates \(energy, gradient\): ([0-9.eE+-]+)", report).group(1))
    assert spread < 1e-10, report
    e, g = eng.energy_and_grad(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert abs(e - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)
    assert "kernel" in eng.describe() or "bwd" in eng.describe()
    eng.close()
    # a second backend of the same shape takes the cached choice without timing
    eng2 = Engine(n, L, h)
    report2 = eng2.autotune(p)
    assert report2.startswith("autotune:\ncached"), report2
    e2, g2 = eng2.energy_and_grad(p)
    assert e2 == e and np.array_equal(g2, g)
    eng2.close()

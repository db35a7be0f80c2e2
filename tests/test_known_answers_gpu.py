"""The reference's published known answers, reproduced on the GPU: 20 plain
gradient-descent steps (stepsize 0.08, seed 7, init 0.3 N(0,1), h=1, L=2)
through the drop-in module, final energy vs the reference CSV."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from gpu_simulation_b200 import RingIsingAdjointBackend, StandaloneBackendConfig

pytestmark = pytest.mark.gpu

DATA = json.loads((Path(__file__).parent / "golden" / "csv_known_answers.json").read_text())


@pytest.mark.parametrize("n", [8, 10, 12, 14, 16, 18, 20, 22, 24])
def test_training_loop_reproduces_reference_final_energy(n):
    proto = DATA["protocol"]
    L = proto["layers"]
    backend = RingIsingAdjointBackend(StandaloneBackendConfig(n, L, proto["field"], "structured_adjoint"))
    rng = np.random.default_rng(proto["seed"])
    params = proto["init_scale"] * rng.standard_normal((L, n, 2))
    for _ in range(proto["steps"]):
        _, g = backend.energy_and_grad(params)
        params = params - proto["stepsize"] * g
    final = backend.energy(params)
    for method, value in DATA["final_energy"][str(n)].items():
        assert abs(final - value) < 1e-9, (n, method, final, value)

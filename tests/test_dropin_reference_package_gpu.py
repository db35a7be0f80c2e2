"""The drop-in claim through the reference's own Python package.

``ring_ising.backends.standalone.RingIsingAdjointBackend`` (reference
ring_ising/backends/standalone/runtime.py:12-85) loads
``standalone_backend._cuda_backend`` by name.  With this repository's
``standalone_backend/`` first on ``sys.path`` that import resolves to the
engine's pybind11 module, and the reference's wrapper, its config validation
and its parameter reshaping run unchanged on top of it.  The result must equal
the reference's own CUDA extension (rebuilt for sm_100a, oracle/_ref) at
1e-10.

The reference's package comes from its offline install into baseline/_ref
(``pip install --target baseline/_ref`` of the reference checkout), or from a
checkout named by the REF environment variable; without either the test is
skipped.
"""

from __future__ import annotations

import importlib
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from tests.refmod import load_reference_module

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _reference_package_dir():
    cands = [ROOT / "baseline" / "_ref"]
    if os.environ.get("REF"):
        cands.append(Path(os.environ["REF"]))
    for c in cands:
        if (c / "ring_ising" / "backends" / "standalone" / "runtime.py").is_file():
            return c
    return None


PKG = _reference_package_dir()
ref = load_reference_module()


@pytest.mark.skipif(PKG is None, reason="the reference's Python package is not installed (baseline/_ref) "
                                        "and REF is unset")
@pytest.mark.skipif(ref is None, reason="oracle/_ref not built (make -C oracle ref)")
def test_reference_wrapper_runs_on_the_engine(monkeypatch):
    # this repository first (its standalone_backend), the reference package after it
    monkeypatch.setattr(sys, "path", [str(ROOT), str(PKG)] + [p for p in sys.path if p not in (str(ROOT),)])
    for name in list(sys.modules):
        if name == "ring_ising" or name.startswith("ring_ising."):
            monkeypatch.delitem(sys.modules, name)
    standalone = importlib.import_module("ring_ising.backends.standalone")
    assert Path(standalone.__file__).resolve().is_relative_to(PKG.resolve())
    mod = importlib.import_module("standalone_backend._cuda_backend")
    assert Path(mod.__file__).resolve().parent == (ROOT / "standalone_backend").resolve()

    n, L, h = 12, 3, 1.0
    cfg = standalone.StandaloneBackendConfig(num_qubits=n, layers=L, field=h,
                                             gradient_strategy="structured_adjoint")
    backend = standalone.RingIsingAdjointBackend(cfg)
    params = np.random.default_rng(7).uniform(0, 2 * np.pi, cfg.param_shape)
    e, g = backend.energy_and_grad(params)
    assert g.shape == cfg.param_shape
    e_only = backend.energy(params)
    prof = backend.profile_energy_and_grad(params)

    r = ref.RingIsingCudaBackend(n, L, h, "structured_adjoint", 8, False).energy_and_grad(
        params.reshape(-1), True, False)
    assert abs(e - r["energy"]) < 1e-10
    assert abs(e_only - r["energy"]) < 1e-10
    np.testing.assert_allclose(g.reshape(-1), np.asarray(r["gradient"]), atol=1e-10, rtol=0)
    np.testing.assert_allclose(prof["gradient"].reshape(-1), np.asarray(r["gradient"]), atol=1e-10, rtol=0)
    assert set(prof["timings_ms"])  # the stage names of the reference's profiler

    # the reference's own validation messages still guard the call
    with pytest.raises(ValueError, match="Expected params with shape"):
        backend.energy(params.reshape(-1))

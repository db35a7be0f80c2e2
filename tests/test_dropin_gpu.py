"""The drop-in module standalone_backend._cuda_backend behaves like the
reference's pybind11 API (cpp/ising_cuda_bindings.cpp:71-144)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_class_api_and_return_dicts():
    import standalone_backend._cuda_backend as m

    n, L, h = 10, 3, 1.1
    p = np.random.default_rng(4).uniform(0, 2 * np.pi, 2 * n * L)
    b = m.RingIsingCudaBackend(num_qubits=n, num_layers=L, field=h)
    r = b.energy_and_grad(p)
    assert set(r) == {"energy", "gradient"}
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert abs(r["energy"] - e_ref) < 1e-10
    np.testing.assert_allclose(r["gradient"], g_ref, atol=1e-10, rtol=0)
    r2 = b.energy_and_grad(p, False)
    assert abs(r2["energy"] - e_ref) < 1e-10
    rp = b.energy_and_grad(p, True, True)
    assert "timings_ms" in rp and "backward_sweep_ms" in rp["timings_ms"]
    np.testing.assert_allclose(rp["gradient"], g_ref, atol=1e-10, rtol=0)
    # array-likes are converted (forcecast), as in the reference
    r3 = b.energy_and_grad(list(p))
    assert r3["energy"] == r["energy"]


def test_module_function_and_graph_benchmark():
    import standalone_backend._cuda_backend as m

    n, L = 12, 2
    p = np.random.default_rng(6).uniform(0, 2 * np.pi, 2 * n * L)
    r = m.energy_and_grad(n, L, 1.0, "structured_adjoint", p)
    e_ref, _ = oracle.energy_and_grad(n, L, 1.0, p)
    assert abs(r["energy"] - e_ref) < 1e-10
    with pytest.raises(ValueError):
        m.energy_and_grad(n, L, 1.0, "structured_adjoint", p.reshape(2, -1))
    with pytest.raises(ValueError):
        m.energy_and_grad(n, L, 1.0, "structured_adjoint", p[:-1])
    b = m.RingIsingCudaBackend(n, L, 1.0)
    bench = b.benchmark_structured_forward_graph(p, 5)
    assert set(bench) == {"normal_forward_ms", "graph_forward_ms", "speedup"}
    with pytest.raises(ValueError):
        b.benchmark_structured_forward_graph(p, 0)


def test_errors_map_to_python_exceptions():
    import standalone_backend._cuda_backend as m

    with pytest.raises(ValueError):
        m.RingIsingCudaBackend(4, 2, 1.0, "no_such_strategy")
    with pytest.raises(ValueError):
        m.RingIsingCudaBackend(4, 2, 1.0, "structured_adjoint", 0)
    b = m.RingIsingCudaBackend(4, 2, 1.0)
    with pytest.raises(ValueError):
        b.energy_and_grad(np.zeros(3))


def test_wrapper_profile_and_shapes():
    from gpu_simulation_b200 import RingIsingAdjointBackend, StandaloneBackendConfig

    cfg = StandaloneBackendConfig(8, 2, 0.9, "structured_adjoint")
    be = RingIsingAdjointBackend(cfg)
    p = np.random.default_rng(1).uniform(0, 2 * np.pi, cfg.param_shape)
    e, g = be.energy_and_grad(p)
    assert g.shape == cfg.param_shape
    prof = be.profile_energy_and_grad(p)
    assert abs(prof["energy"] - e) < 1e-13
    with pytest.raises(ValueError):
        be.energy(np.zeros((2, 8)))

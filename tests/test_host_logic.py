"""Host logic of the engine without a GPU: the C ABI library loads and exports
every entry point of include/rsv.h, the pass plan executed in numpy equals
the oracle, the ring maps equal the reference's closed form, and invalid
arguments are rejected before any device call."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import _lib, describe_plan
from tests import plan_sim

ROOT = Path(__file__).resolve().parent.parent


def declared_functions() -> list[str]:
    names = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names.update(re.findall(r"\b(rsv_[a-z_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.load_library()
    names = declared_functions()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib._SIGNATURES, f"{name} has no ctypes signature"


def test_dropin_module_exports_reference_api():
    import standalone_backend._cuda_backend as m

    assert hasattr(m, "RingIsingCudaBackend")
    assert hasattr(m, "energy_and_grad")
    cls = m.RingIsingCudaBackend
    assert hasattr(cls, "energy_and_grad")
    assert hasattr(cls, "benchmark_structured_forward_graph")


def test_ring_map_matches_oracle_closed_form():
    lib = _lib.load_library()
    rng = np.random.default_rng(1)
    for n in (2, 3, 5, 12, 20, 28, 31):
        for i in rng.integers(0, 1 << n, 64):
            i = int(i)
            assert lib.rsv_ring_map(i, n, 0) == oracle.ring_perm(i, n)
            assert lib.rsv_ring_map(i, n, 1) == oracle.ring_perm(i, n, inverse=True)


@pytest.mark.parametrize("n,L,h", [
    (2, 1, 0.7), (2, 3, 1.0), (3, 2, 1.1), (5, 4, 0.3), (8, 2, 1.0), (11, 2, 0.9),
    (12, 3, 1.0), (13, 1, 1.2), (13, 3, 0.8), (14, 2, 1.0), (16, 2, 2.0), (17, 2, 0.5),
    (13, 4, 0.8), (14, 5, 1.1),
])
def test_plan_executed_in_numpy_matches_oracle(n, L, h):
    rng = np.random.default_rng(100 + n * 10 + L)
    p = rng.uniform(0, 2 * np.pi, 2 * n * L)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    for mode in (plan_sim.UNCOMPUTE, plan_sim.CHECKPOINT):
        e_sim, g_sim = plan_sim.simulate(n, L, h, p, mode=mode)
        assert abs(e_sim - e_ref) < 1e-11
        np.testing.assert_allclose(g_sim, g_ref, atol=1e-11, rtol=0)


@pytest.mark.parametrize("n,L", [(20, 4), (24, 4), (28, 4), (30, 4), (31, 2), (28, 9)])
def test_large_plans_cover_every_wire_once(n, L):
    for mode in (plan_sim.AUTO, plan_sim.UNCOMPUTE, plan_sim.CHECKPOINT):
        plan = plan_sim.parse_plan(plan_sim.describe_plan(n, L, mode))
        check_large_plan(plan, n, L)
    # automatic choice: the checkpoint schedule while its buffers fit 128 GiB
    auto = plan_sim.parse_plan(describe_plan(n, L))
    ck = plan_sim.parse_plan(plan_sim.describe_plan(n, L, plan_sim.CHECKPOINT))
    fits = ck["bufs"] * 16 * 2 ** n <= 128 * 2 ** 30
    assert auto["mode"] == ("checkpoint" if fits else "uncompute")
    # uncompute: psi, lambda and the target of the inverse-ring scatter (not
    # needed when the leading layers are one read of lambda)
    assert plan_sim.parse_plan(plan_sim.describe_plan(n, L, plan_sim.UNCOMPUTE))["bufs"] in (2, 3)


def check_large_plan(plan, n, L):
    seen = {}
    for st in plan["steps"]:
        if st.get("kind") == "mps_fwd":
            assert 0 <= st["out"] < plan["bufs"]
            continue
        for b in ("psi_in", "psi_out", "lam_in", "lam_out"):
            assert -1 <= st[b] < plan["bufs"]
        if plan["mode"] == "checkpoint" and st["bwd"]:
            assert st["psi_store"] == "none"
        if st["bwd"]:
            for w in st["gates"]:
                key = (st["layer"], w)
                assert key not in seen
                seen[key] = st["pass_index"]
    # buffer ids are compact: every id below bufs is used (at least two buffers)
    used = {plan["energy"][0], plan["energy"][1]}
    for st in plan["steps"]:
        if st.get("kind") == "mps_fwd":
            used.add(st["out"])
            continue
        used.update(b for b in (st["psi_in"], st["psi_out"], st["lam_in"], st["lam_out"]) if b >= 0)
    if plan["mps"] is not None:
        used.add(plan["mps"]["buf"])
    if plan["layer0"] is not None:
        used.add(plan["layer0"]["buf"])
    assert used == set(range(max(len(used), 2))) and plan["bufs"] == max(len(used), 2)
    if plan["mps"] is not None:
        # the first K layers are one read of lambda on the matrix-product kernels
        K = plan["mps"]["K"]
        assert all(layer >= K for layer, _ in seen)
        assert 0 <= plan["mps"]["buf"] < plan["bufs"]
        fwd = [st for st in plan["steps"] if st.get("kind") != "mps_fwd" and not st["bwd"]]
        if K == 3 and L > K:
            # the bond-4 state is evaluated by layer 3's first forward pass itself
            assert not any(st.get("kind") == "mps_fwd" for st in plan["steps"])
            assert fwd[0]["psi_load"] == "mpsP" and fwd[0]["layer"] == K
        bwd = [st for st in plan["steps"] if st.get("kind") != "mps_fwd" and st["bwd"]]
        if bwd:
            # psi below layer K is never needed
            assert bwd[-1]["psi_store"] == "none"
        for layer in range(K):
            for w in range(n):
                seen[(layer, w)] = -1
    if plan["layer0"] is not None:
        # layer 0 is one read of lambda on the layer-0 kernel, no backward pass
        assert all(layer != 0 for layer, _ in seen)
        assert 0 <= plan["layer0"]["buf"] < plan["bufs"]
        for w in range(n):
            seen[(0, w)] = -1
    assert len(seen) == n * L
    # at most three backward passes per layer for these sizes
    bwd = [s for s in plan["steps"] if s.get("bwd")]
    assert len(bwd) <= 3 * L


def test_plan_rejects_bad_shapes():
    with pytest.raises(ValueError):
        describe_plan(1, 2)
    with pytest.raises(ValueError):
        describe_plan(32, 2)
    with pytest.raises(ValueError):
        describe_plan(8, 0)


@pytest.mark.parametrize("kwargs,msg", [
    (dict(num_qubits=1, num_layers=2, strategy="structured_adjoint", width=8), "num_qubits"),
    (dict(num_qubits=4, num_layers=0, strategy="structured_adjoint", width=8), "num_layers"),
    (dict(num_qubits=4, num_layers=2, strategy="checkpoint", width=8), "Unknown gradient strategy"),
    (dict(num_qubits=4, num_layers=2, strategy="structured_adjoint", width=0), "at least 1"),
    (dict(num_qubits=4, num_layers=2, strategy="structured_adjoint", width=9), "exceeds"),
    (dict(num_qubits=9, num_layers=2, strategy="dense_scan", width=8), "dense_scan"),
])
def test_create_validates_arguments_before_touching_the_gpu(kwargs, msg):
    lib = _lib.load_library()
    h = ctypes.c_void_p()
    rc = lib.rsv_create(kwargs["num_qubits"], kwargs["num_layers"], 1.0, kwargs["strategy"].encode(),
                        kwargs["width"], 0, ctypes.byref(h))
    assert rc == _lib.RSV_ERR_INVALID_ARGUMENT
    assert msg in lib.rsv_last_error().decode()
    assert not h.value


def test_null_backend_calls_are_rejected():
    lib = _lib.load_library()
    e = ctypes.c_double()
    rc = lib.rsv_energy_and_grad(None, None, 0, 1, ctypes.byref(e), None, None)
    assert rc == _lib.RSV_ERR_INVALID_ARGUMENT
    assert lib.rsv_destroy(None) == 0


def test_batch_sharding_and_synthetic_batch():
    from gpu_simulation_b200.batch import circuit_cost, param_offsets, shard_circuits, synthetic_batch

    ns, ls, hs, params = synthetic_batch(count=300, seed=7)
    assert ns.min() >= 6 and ns.max() <= 16 and ls.min() >= 1 and ls.max() <= 16
    assert np.all((hs >= 0.2) & (hs < 2.0))
    assert params.size == param_offsets(ns, ls)[-1]
    ns2, ls2, hs2, params2 = synthetic_batch(count=300, seed=7)
    assert np.array_equal(ns, ns2) and np.array_equal(params, params2)
    cost = circuit_cost(ns, ls)
    for world in (1, 2, 3, 8):
        parts = shard_circuits(ns, ls, world)
        assert len(parts) == world
        assert np.array_equal(np.concatenate(parts), np.arange(ns.size))
        if world > 1:
            loads = np.array([cost[p].sum() for p in parts])
            assert loads.max() - loads.min() <= 2 * cost.max()


def test_initial_params_follow_the_reference_recipe():
    from gpu_simulation_b200.training import make_initial_params

    p = make_initial_params(8, 2, 7, 0.3)
    assert p.shape == (2, 8, 2) and p.dtype == np.float64
    np.testing.assert_array_equal(p, 0.3 * np.random.default_rng(7).standard_normal((2, 8, 2)))


def test_device_optimiser_steps_reject_bad_arguments_before_any_launch():
    # argument checks of the device-resident update steps run on the host
    lib = _lib.load_library()
    fake = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    assert lib.rsv_adam_vqe_step_f64(None, fake, fake, fake, 4, 0.05, 0.9, 0.999, 1e-8, fake, None, fake,
                                     None) == _lib.RSV_ERR_INVALID_ARGUMENT
    assert lib.rsv_adam_vqe_step_f64(fake, fake, fake, fake, 4, float("nan"), 0.9, 0.999, 1e-8, fake, None,
                                     fake, None) == _lib.RSV_ERR_INVALID_ARGUMENT
    assert lib.rsv_adam_vqe_step_f64(fake, fake, fake, fake, 4, 0.05, 1.0, 0.999, 1e-8, fake, None, fake,
                                     None) == _lib.RSV_ERR_INVALID_ARGUMENT
    assert lib.rsv_gd_step_f64(fake, None, 4, 0.1, fake, None, None, fake, None) == _lib.RSV_ERR_INVALID_ARGUMENT


def test_kernel_launch_counter_rejects_null_arguments():
    lib = _lib.load_library()
    out = ctypes.c_ulonglong()
    assert lib.rsv_kernel_launches(None, ctypes.byref(out)) == _lib.RSV_ERR_INVALID_ARGUMENT


def test_plan_invariants_over_every_size():
    # every wire once, compact buffer ids, the fused bond-4 source and no psi
    # store below the matrix-product layers, for all multi-tile sizes
    for n in range(13, 32):
        for L in range(1, 7):
            for mode in (plan_sim.AUTO, plan_sim.UNCOMPUTE, plan_sim.CHECKPOINT):
                plan = plan_sim.parse_plan(plan_sim.describe_plan(n, L, mode))
                check_large_plan(plan, n, L)

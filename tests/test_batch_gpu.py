"""Batched circuits (rsv_batch_*): every circuit of a mixed batch against the
CPU oracle at 1e-10, against the single-circuit engine, slot reuse across
circuit sizes, the energy-only path, CUDA-graph replay and argument checks."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import BatchEngine, Engine
from gpu_simulation_b200.batch import param_offsets, synthetic_batch

pytestmark = pytest.mark.gpu

TOL = 1e-10


def mixed_batch(seed=3):
    # every qubit count 2..16 (padded, single-tile, 2/3-pass layouts) with a few depths
    rng = np.random.default_rng(seed)
    ns, ls = [], []
    for n in range(2, 17):
        for L in (1, 2, 5):
            ns.append(n)
            ls.append(L)
    ns += [16, 13, 12, 7]
    ls += [16, 9, 11, 16]
    ns = np.array(ns, dtype=np.int32)
    ls = np.array(ls, dtype=np.int32)
    perm = rng.permutation(ns.size)
    ns, ls = ns[perm], ls[perm]
    hs = rng.uniform(0.2, 2.0, ns.size)
    params = rng.uniform(0.0, 2.0 * np.pi, int(param_offsets(ns, ls)[-1]))
    return ns, ls, hs, params


def check_against_oracle(ns, ls, hs, params, e, g, which):
    off = param_offsets(ns, ls)
    for c in which:
        n, L, h = int(ns[c]), int(ls[c]), float(hs[c])
        p = params[off[c]:off[c + 1]]
        e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
        assert abs(e[c] - e_ref) < TOL, (c, n, L, e[c], e_ref)
        np.testing.assert_allclose(g[off[c]:off[c + 1]], g_ref, atol=TOL, rtol=0,
                                   err_msg=f"circuit {c} n={n} L={L}")


def test_mixed_batch_matches_oracle():
    ns, ls, hs, params = mixed_batch()
    e, g = BatchEngine().energy_and_grad(ns, ls, hs, params)
    check_against_oracle(ns, ls, hs, params, e, g, range(ns.size))


def test_slot_reuse_small_after_large():
    # two circuits in flight: every slot runs many circuits of different sizes
    # (a padded n < 12 circuit after an n = 16 one must not see stale data)
    ns, ls, hs, params = mixed_batch(seed=11)
    eng = BatchEngine(slots=2)
    e, g = eng.energy_and_grad(ns, ls, hs, params)
    check_against_oracle(ns, ls, hs, params, e, g, range(ns.size))
    eng.set_active_slots(1)
    e1, g1 = eng.energy_and_grad(ns, ls, hs, params)
    assert np.array_equal(e, e1) and np.array_equal(g, g1)


def test_matches_single_circuit_engine():
    ns, ls, hs, params = mixed_batch(seed=5)
    e, g = BatchEngine().energy_and_grad(ns, ls, hs, params)
    off = param_offsets(ns, ls)
    for c in range(0, ns.size, 3):
        es, gs = Engine(int(ns[c]), int(ls[c]), float(hs[c])).energy_and_grad(params[off[c]:off[c + 1]])
        assert abs(e[c] - es) < 1e-12
        np.testing.assert_allclose(g[off[c]:off[c + 1]], gs, atol=1e-12, rtol=0)


def test_energy_only_and_determinism():
    ns, ls, hs, params = mixed_batch(seed=8)
    eng = BatchEngine()
    e, g = eng.energy_and_grad(ns, ls, hs, params)
    e2, g2 = eng.energy_and_grad(ns, ls, hs, params)
    assert np.array_equal(e, e2) and np.array_equal(g, g2)
    e3, none = eng.energy_and_grad(ns, ls, hs, params, compute_gradient=False)
    assert none is None
    assert np.array_equal(e, e3)


def test_device_run_and_graph_replay():
    import torch

    ns, ls, hs, params = synthetic_batch(count=512, seed=7)
    eng = BatchEngine()
    eng.set_circuits(ns, ls, hs)
    dev = torch.device("cuda", 0)
    p = torch.from_numpy(params).to(dev)
    e = torch.empty(ns.size, dtype=torch.float64, device=dev)
    g = torch.empty_like(p)
    eng.run_device(p, e, g)
    torch.cuda.synchronize()
    e_host, g_host = BatchEngine().energy_and_grad(ns, ls, hs, params)
    assert np.array_equal(e.cpu().numpy(), e_host)
    assert np.array_equal(g.cpu().numpy(), g_host)
    graph = eng.capture_graph(p, e, g)
    e.zero_()
    g.zero_()
    p2 = torch.from_numpy(synthetic_batch(count=512, seed=7)[3] * 0.5).to(dev)
    p.copy_(p2)
    graph.replay()
    torch.cuda.synchronize()
    e_ref, g_ref = BatchEngine().energy_and_grad(ns, ls, hs, p2.cpu().numpy())
    assert np.array_equal(e.cpu().numpy(), e_ref)
    assert np.array_equal(g.cpu().numpy(), g_ref)
    # a sample against the oracle
    check_against_oracle(ns, ls, hs, p2.cpu().numpy(), e_ref, g_ref, range(0, 512, 37))


def test_full_size_batch_sample_and_variational_bound():
    ns, ls, hs, params = synthetic_batch(count=4096, seed=7)
    e, g = BatchEngine().energy_and_grad(ns, ls, hs, params)
    assert np.all(np.isfinite(e)) and np.all(np.isfinite(g))
    # |E| <= ||H|| <= n (1 + h)
    assert np.all(np.abs(e) <= ns * (1.0 + hs) + 1e-9)
    rng = np.random.default_rng(0)
    check_against_oracle(ns, ls, hs, params, e, g, rng.choice(ns.size, 24, replace=False))


def test_invalid_arguments():
    eng = BatchEngine(max_qubits=12)
    with pytest.raises(ValueError):
        eng.set_circuits([13], [2], [1.0])
    with pytest.raises(ValueError):
        eng.set_circuits([8], [65], [1.0])
    with pytest.raises(ValueError):
        eng.set_circuits([1], [2], [1.0])
    with pytest.raises(ValueError):
        eng.set_circuits([8, 9], [2], [1.0])
    with pytest.raises(ValueError):
        eng.energy_and_grad([8], [2], [1.0], np.zeros(5))
    with pytest.raises(ValueError):
        eng.set_active_slots(0)
    with pytest.raises(ValueError):
        BatchEngine(max_qubits=17)
    e, g = eng.energy_and_grad([], [], [], np.zeros(0))
    assert e.size == 0 and g.size == 0


def test_cluster_sizes_agree():
    # circuits spread over 1, 2, 4 or 8 CTAs of a thread-block cluster (tiles
    # split between them, sums added through distributed shared memory) give
    # the same energies and gradients to rounding, each matching the oracle
    ns, ls, hs, params = mixed_batch(seed=21)
    eng = BatchEngine()
    info = eng.cluster()
    assert info["cluster"] in (1, 2, 4, 8) and info["max_active_clusters"] >= 1
    results = {}
    for c in (1, 2, 4, 8):
        eng.set_cluster(c)
        assert eng.cluster()["cluster"] == c
        results[c] = eng.energy_and_grad(ns, ls, hs, params)
        e2, g2 = eng.energy_and_grad(ns, ls, hs, params)
        assert np.array_equal(results[c][0], e2) and np.array_equal(results[c][1], g2)
    for c in (2, 4, 8):
        np.testing.assert_allclose(results[c][0], results[1][0], atol=1e-12, rtol=0)
        np.testing.assert_allclose(results[c][1], results[1][1], atol=1e-12, rtol=0)
    e, g = results[8]
    check_against_oracle(ns, ls, hs, params, e, g, range(ns.size))
    with pytest.raises(ValueError):
        eng.set_cluster(3)

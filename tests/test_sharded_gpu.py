"""Sharded single circuit on the GPU: each CUDA kernel of include/rsv_shard.h
against its numpy restatement (tests/shard_numpy_ops.py) on the same inputs,
and ``ShardedEngine`` with 1, 2, 4 and 8 virtual ranks on one GPU against the
oracle and the single-GPU engine.  (This run has one GPU: the NCCL exchange of
real ranks is the same schedule, checked with two gloo processes on CPU in
test_sharded.py.)
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine
from gpu_simulation_b200.sharded import CudaShardOps, ShardedEngine
from tests.shard_numpy_ops import NumpyShardOps

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GEOMETRIES = [(12, 0), (14, 1), (16, 2), (18, 3)]


def _rand_state(rng, size):
    return torch.from_numpy(rng.standard_normal(size) + 1j * rng.standard_normal(size))


def _pair(t):
    """A CPU copy and a CUDA copy of the same tensor."""
    return t.clone(), t.clone().cuda()


def _close(gpu, cpu, tol=1e-13):
    """Equal to rounding, relative to the vector's largest entry (the forward
    gates scale the state by 1/f per gate)."""
    c = cpu.numpy()
    np.testing.assert_allclose(gpu.cpu().numpy(), c, atol=tol * max(1.0, float(np.max(np.abs(c)))), rtol=0)


def _coefs(rng, n, L):
    p = torch.from_numpy(rng.uniform(0, 2 * np.pi, 2 * n * L))
    c_cpu = torch.zeros(4 * n * L, dtype=torch.float64)
    NumpyShardOps().coef(n, L, p, c_cpu)
    c_gpu = torch.zeros(4 * n * L, dtype=torch.float64, device="cuda")
    CudaShardOps().coef(n, L, p.cuda(), c_gpu)
    torch.cuda.synchronize()
    np.testing.assert_allclose(c_gpu.cpu().numpy(), c_cpu.numpy(), atol=1e-15, rtol=0)
    return c_cpu, c_gpu


@pytest.mark.parametrize("n,g", GEOMETRIES)
def test_kernels_match_numpy_restatement(n, g):
    rng = np.random.default_rng(300 + n + g)
    L = 3
    layer = 1
    N, local = 1 << g, 1 << (n - g)
    npo, cuo = NumpyShardOps(), CudaShardOps()
    c_cpu, c_gpu = _coefs(rng, n, L)
    scratch = torch.zeros(cuo.scratch_doubles(n, g), dtype=torch.float64, device="cuda")
    for rank in range(N):
        # local rotations and their adjoint
        a_cpu, a_gpu = _pair(_rand_state(rng, local))
        npo.rotate_local(n, g, layer, c_cpu, a_cpu)
        cuo.rotate_local(n, g, layer, c_gpu, a_gpu)
        _close(a_gpu, a_cpu)
        l_cpu, l_gpu = _pair(_rand_state(rng, local))
        r_cpu = torch.zeros(2 + 2 * n * L, dtype=torch.float64)
        r_gpu = r_cpu.clone().cuda()
        npo.rotate_local_adjoint(n, g, L, layer, c_cpu, a_cpu, l_cpu, None, r_cpu)
        cuo.rotate_local_adjoint(n, g, L, layer, c_gpu, a_gpu, l_gpu, scratch, r_gpu)
        _close(a_gpu, a_cpu)
        _close(l_gpu, l_cpu)
        _close(r_gpu, r_cpu, 1e-12)
        # energy terms of the local wires
        npo.energy_local(n, g, rank, 0.9, a_cpu, l_cpu, None, r_cpu)
        cuo.energy_local(n, g, rank, 0.9, a_gpu, l_gpu, scratch, r_gpu)
        _close(l_gpu, l_cpu)
        assert abs(r_gpu[0].item() - r_cpu[0].item()) < 1e-12 * abs(r_cpu[0].item()) + 1e-9
        # forward ring exchange, both sides (permutations: bit-exact)
        s_cpu, s_gpu = _pair(_rand_state(rng, local))
        o_cpu, o_gpu = _pair(torch.zeros(local, dtype=torch.complex128))
        npo.ring_pack(n, g, rank, layer, c_cpu, s_cpu, o_cpu)
        cuo.ring_pack(n, g, rank, layer, c_gpu, s_gpu, o_gpu)
        _close(o_gpu, o_cpu)
        npo.ring_unpack(n, g, rank, s_cpu, o_cpu)
        cuo.ring_unpack(n, g, rank, s_gpu, o_gpu)
        assert np.array_equal(o_gpu.cpu().numpy(), o_cpu.numpy())
        # backward ring exchange
        p_cpu, p_gpu = _pair(_rand_state(rng, local))
        q_cpu, q_gpu = _pair(_rand_state(rng, local))
        sp_cpu, sp_gpu = _pair(torch.zeros(local, dtype=torch.complex128))
        sl_cpu, sl_gpu = _pair(torch.zeros(local, dtype=torch.complex128))
        npo.ring_pack_adjoint(n, g, rank, p_cpu, q_cpu, sp_cpu, sl_cpu)
        cuo.ring_pack_adjoint(n, g, rank, p_gpu, q_gpu, sp_gpu, sl_gpu)
        assert np.array_equal(sp_gpu.cpu().numpy(), sp_cpu.numpy())
        assert np.array_equal(sl_gpu.cpu().numpy(), sl_cpu.numpy())
        for add_field, lay in ((True, layer), (False, layer), (True, -1)):
            r_cpu.zero_()
            r_gpu.zero_()
            npo.ring_unpack_adjoint(n, g, rank, L, lay, c_cpu, 1.2, add_field, p_cpu, q_cpu, sp_cpu, sl_cpu, None,
                                    r_cpu)
            cuo.ring_unpack_adjoint(n, g, rank, L, lay, c_gpu, 1.2, add_field, p_gpu, q_gpu, sp_gpu, sl_gpu, scratch,
                                    r_gpu)
            _close(sp_gpu, sp_cpu)
            _close(sl_gpu, sl_cpu)
            _close(r_gpu, r_cpu, 1e-12)


@pytest.mark.parametrize("n,L,h,ranks", [(12, 3, 0.7, 1), (14, 2, 1.1, 2), (16, 3, 0.9, 4), (18, 2, 1.3, 8),
                                         (19, 4, 1.0, 8)])
def test_virtual_ranks_match_oracle(n, L, h, ranks):
    p = np.random.default_rng(500 + n).uniform(0, 2 * np.pi, 2 * n * L)
    eng = ShardedEngine(n, L, h, virtual_ranks=ranks)
    e, g = eng.energy_and_grad(p)
    e2, g2 = eng.energy_and_grad(p)
    e_only = eng.energy(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert e == e2 and np.array_equal(g, g2)  # fixed-order sums
    assert abs(e - e_ref) < 1e-10 and abs(e_only - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


def test_many_layers_keep_their_scale():
    """Forward gates run in tangent form ((1/f) RY, f >= 1/sqrt(2)); each
    layer's ring exchange restores the layer's prod f, so 96 layers with every
    theta near pi/2 (the largest 1/f) neither overflow nor lose accuracy."""
    n, L, h, ranks = 14, 96, 0.9, 2
    rng = np.random.default_rng(96)
    p = rng.uniform(0, 2 * np.pi, (L, n, 2))
    p[..., 0] = np.pi / 2 + rng.uniform(-0.01, 0.01, (L, n))
    p = p.reshape(-1)
    e, g = ShardedEngine(n, L, h, virtual_ranks=ranks).energy_and_grad(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert np.isfinite(e) and abs(e - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


@pytest.mark.parametrize("n,L,h,ranks", [(24, 4, 1.0, 4), (26, 4, 0.8, 8), (28, 4, 1.0, 2)])
def test_virtual_ranks_match_single_gpu_engine(n, L, h, ranks):
    p = np.random.default_rng(7).uniform(0, 2 * np.pi, 2 * n * L)
    eng = Engine(n, L, h)
    try:
        e_ref, g_ref = eng.energy_and_grad(p)
    finally:
        eng.close()
    torch.cuda.empty_cache()
    sh = ShardedEngine(n, L, h, virtual_ranks=ranks)
    e, g = sh.energy_and_grad(p)
    del sh
    torch.cuda.empty_cache()
    assert abs(e - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


def test_cuda_ops_refuse_cpu_tensors():
    with pytest.raises(ValueError):
        CudaShardOps().init(12, 0, 0, torch.zeros(4096, dtype=torch.complex128))


def test_edge_cases_and_successive_calls():
    """h = 0 and L = 1, parameters as a CUDA tensor, and calls with different
    angles in a row on the same engine (every call starts from |0...0>)."""
    n = 16
    for L, h, ranks in ((1, 0.0, 4), (3, 1.2, 2)):
        eng = ShardedEngine(n, L, h, virtual_ranks=ranks)
        for seed in (1, 2):
            p = np.random.default_rng(seed).uniform(0, 2 * np.pi, 2 * n * L)
            e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
            e, g = eng.energy_and_grad(torch.tensor(p, device="cuda"))
            assert abs(e - e_ref) < 1e-10
            np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)
            assert abs(eng.energy(p) - e_ref) < 1e-10


def test_autograd_function_matches_single_gpu_autograd():
    from gpu_simulation_b200 import ring_ising_energy
    from gpu_simulation_b200.sharded import sharded_ring_ising_energy

    n, L, h = 16, 3, 0.8
    p0 = np.random.default_rng(31).uniform(0, 2 * np.pi, (L, n, 2))
    a = torch.tensor(p0, device="cuda", requires_grad=True)
    b = torch.tensor(p0, device="cuda", requires_grad=True)
    eng = Engine(n, L, h)
    try:
        ea = ring_ising_energy(a, eng)
        ea.backward()
    finally:
        eng.close()
    eb = sharded_ring_ising_energy(b, ShardedEngine(n, L, h, virtual_ranks=4))
    eb.backward()
    assert abs(float(ea.detach()) - float(eb.detach())) < 1e-10
    np.testing.assert_allclose(b.grad.cpu().numpy(), a.grad.cpu().numpy(), atol=1e-10, rtol=0)

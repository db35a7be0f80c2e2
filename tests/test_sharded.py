"""Sharded single circuit on CPU: the exchange schedule of ``ShardedEngine``
(layouts C and S, the ring all-to-all, the rank-ordered sums) with the numpy
restatement of the per-rank operations, against the oracle; as virtual ranks
in one process and as two ``gloo`` processes.  The CUDA kernels of the same
operations are checked against this restatement in test_sharded_gpu.py.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import _lib
from tests.shard_numpy_ops import Geometry, NumpyShardOps, ring_map, ring_map_inv

torch = pytest.importorskip("torch")


def _engine(n, L, h, ranks):
    from gpu_simulation_b200.sharded import ShardedEngine

    return ShardedEngine(n, L, h, virtual_ranks=ranks, device="cpu", ops=NumpyShardOps())


def test_ring_map_matches_oracle():
    rng = np.random.default_rng(5)
    for n in (12, 14, 20, 33):
        xs = rng.integers(0, 1 << n, size=64, dtype=np.uint64)
        ys = ring_map(xs, n)
        for x, y in zip(xs.tolist(), ys.tolist()):
            assert oracle.ring_perm(int(x), n) == y
        assert np.array_equal(ring_map_inv(ys, n), xs)


def test_layouts_partition_the_index_space():
    n, g = 16, 2
    G = Geometry(n, g)
    for layout in ("c", "s"):
        seen = np.concatenate([getattr(G, "global_" + layout)(r) for r in range(G.N)])
        assert np.array_equal(np.sort(seen), np.arange(1 << n, dtype=np.uint64))
    # C -> S is the all-to-all of 2^(n-2g) blocks: block j of rank r (C)
    # holds exactly the amplitudes that rank j (S) keeps at block r
    for r in range(G.N):
        xc = G.global_c(r).reshape(G.N, G.B)
        for j in range(G.N):
            xs = G.global_s(j).reshape(G.N, G.B)
            assert np.array_equal(xc[j], xs[r])


@pytest.mark.parametrize("n,L,h,ranks", [(12, 2, 0.7, 1), (14, 2, 1.1, 2), (16, 2, 0.9, 4), (18, 1, 1.3, 8)])
def test_virtual_ranks_match_oracle(n, L, h, ranks):
    p = np.random.default_rng(40 + n).uniform(0, 2 * np.pi, 2 * n * L)
    eng = _engine(n, L, h, ranks)
    e, g = eng.energy_and_grad(p)
    e_only = eng.energy(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert abs(e - e_ref) < 1e-10 and abs(e_only - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


def test_geometry_checks():
    lib = _lib.load_library()
    assert lib.rsv_shard_check(33, 3) == 0
    assert lib.rsv_shard_check(34, 3) == 0
    assert lib.rsv_shard_check(17, 3) == _lib.RSV_ERR_INVALID_ARGUMENT  # n - 2g < 12
    assert "at least 12" in lib.rsv_last_error().decode()
    assert lib.rsv_shard_check(33, 1) == _lib.RSV_ERR_INVALID_ARGUMENT  # 2^32 amplitudes per rank
    assert lib.rsv_shard_check(20, 4) == _lib.RSV_ERR_INVALID_ARGUMENT
    assert lib.rsv_shard_scratch_doubles(17, 3) == 0
    with pytest.raises(ValueError):
        _engine(14, 1, 1.0, 3)  # not a power of two


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, n, L, h, p, out):
    import torch.distributed as dist

    from gpu_simulation_b200.sharded import ShardedEngine

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        eng = ShardedEngine(n, L, h, group=dist.group.WORLD, device="cpu", ops=NumpyShardOps())
        e, g = eng.energy_and_grad(p)
        out.put((rank, e, g))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_oracle():
    import torch.multiprocessing as mp

    n, L, h = 14, 2, 0.8
    p = np.random.default_rng(77).uniform(0, 2 * np.pi, 2 * n * L)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, n, L, h, p, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    results = [out.get(timeout=120) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    (_, e0, g0), (_, e1, g1) = sorted(results, key=lambda t: t[0])
    assert e0 == e1 and np.array_equal(g0, g1)  # every rank returns the same sums
    assert abs(e0 - e_ref) < 1e-10
    np.testing.assert_allclose(g0, g_ref, atol=1e-10, rtol=0)


def _prefix_xor(t, g):
    t = t ^ (t << 1)
    t = t ^ (t << 2)
    return t & ((1 << g) - 1)


def _prefix_inv(z, g):
    return (z ^ (z << 1)) & ((1 << g) - 1)


@pytest.mark.parametrize("n,g", [(12, 0), (14, 1), (16, 2), (18, 3), (19, 3)])
def test_kernel_index_arithmetic(n, g):
    """The closed forms the ring kernels use (rsv_shard.cu) against the index
    maps: destination rank of the forward pack, source of the unpack, and the
    top bits the backward pack solves for, with every index inside its buffer."""
    G = Geometry(n, g)
    N, B, nloc = G.N, G.B, G.nloc
    full = (1 << n) - 1
    u = np.arange(B, dtype=np.int64)
    par_u = np.array([bin(int(x)).count("1") & 1 for x in u])
    for rank in range(N):
        # forward pack (layout S): x = (u, rank, t) goes to rank_C(P(x)) at position u
        for t in range(N):
            x = (u | (rank << (n - 2 * g)) | (t << nloc)).astype(np.uint64)
            pi = par_u ^ (bin(rank).count("1") & 1)
            rd = _prefix_xor(t, g) ^ np.where(pi == 1, N - 1, 0)
            assert np.array_equal(rd, G.rank_c(ring_map(x, n)))
            # backward pack: the t that sends x to this rank
            t_back = _prefix_inv(rd ^ np.where(pi == 1, N - 1, 0), g)
            assert np.all(t_back == t)
        # forward unpack (layout C): closed-form P^-1
        y = G.global_c(rank).astype(np.int64)
        x = ((y ^ (y << 1)) & full) ^ np.where((y >> (n - 1)) & 1 == 1, 3, 0)
        assert np.array_equal(x.astype(np.uint64), ring_map_inv(y.astype(np.uint64), n))
        src = ((x >> (n - 2 * g)) & (N - 1)) * B + (x & (B - 1))
        assert src.min() >= 0 and src.max() < N * B
        assert np.unique(src).size == src.size


def test_many_layers_keep_their_scale():
    """The tangent-form gates scale each layer by prod 1/f; the ring exchange
    restores it, so 96 layers of theta near pi/2 stay finite and exact."""
    n, L, h = 14, 96, 0.9
    rng = np.random.default_rng(96)
    p = rng.uniform(0, 2 * np.pi, (L, n, 2))
    p[..., 0] = np.pi / 2 + rng.uniform(-0.01, 0.01, (L, n))
    p = p.reshape(-1)
    e, g = _engine(n, L, h, 2).energy_and_grad(p)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    assert np.isfinite(e) and abs(e - e_ref) < 1e-10
    np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


def test_edge_cases_and_successive_calls():
    """h = 0 and L = 1, parameters as a tensor, and calls with different angles
    in a row on the same engine (every call starts from |0...0>)."""
    n = 16
    for L, h, ranks in ((1, 0.0, 4), (3, 1.2, 2)):
        eng = _engine(n, L, h, ranks)
        for seed in (1, 2):
            p = np.random.default_rng(seed).uniform(0, 2 * np.pi, 2 * n * L)
            e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
            e, g = eng.energy_and_grad(torch.tensor(p))
            assert abs(e - e_ref) < 1e-10
            np.testing.assert_allclose(g, g_ref, atol=1e-10, rtol=0)


def test_autograd_function_and_adam_step():
    """sharded_ring_ising_energy: gradient through torch autograd equals the
    oracle's, and a torch Adam step runs on it."""
    from gpu_simulation_b200.sharded import sharded_ring_ising_energy

    n, L, h = 14, 2, 1.0
    p0 = np.random.default_rng(3).uniform(0, 2 * np.pi, (L, n, 2))
    eng = _engine(n, L, h, 2)
    params = torch.tensor(p0, requires_grad=True)
    e = sharded_ring_ising_energy(params, eng)
    e.backward()
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p0.reshape(-1))
    assert abs(float(e.detach()) - e_ref) < 1e-10
    np.testing.assert_allclose(params.grad.numpy().reshape(-1), g_ref, atol=1e-10, rtol=0)
    opt = torch.optim.Adam([params], lr=0.05)
    for _ in range(3):
        opt.zero_grad()
        sharded_ring_ising_energy(params, eng).backward()
        opt.step()
    e_after = float(sharded_ring_ising_energy(params, eng).detach())
    assert e_after < e_ref  # three descent steps lower the energy

"""Multi-rank path of the batched circuits on CPU (gloo, world size 2): every
rank takes its cost-balanced contiguous shard, and the final gather rebuilds
the energies and packed gradients in circuit order.  The per-circuit values
are stand-ins computed on the host (the gather is what is tested here)."""

from __future__ import annotations

import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from gpu_simulation_b200.batch import gather_sharded, param_offsets, shard_circuits, synthetic_batch


def fake_results(ns, ls, params):
    off = param_offsets(ns, ls)
    e = np.array([params[off[c]:off[c + 1]].sum() for c in range(ns.size)])
    return e, np.cos(params)


def worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ns, ls, hs, params = synthetic_batch(count=200, seed=7)
        off = param_offsets(ns, ls)
        shards = shard_circuits(ns, ls, world)
        mine = shards[rank]
        lo, hi = (off[mine[0]], off[mine[-1] + 1]) if len(mine) else (0, 0)
        e, g = fake_results(ns[mine], ls[mine], params[lo:hi])
        energy, grad = gather_sharded(torch.from_numpy(e), torch.from_numpy(g), shards, off)
        e_all, g_all = fake_results(ns, ls, params)
        out[rank] = bool(np.array_equal(energy.numpy(), e_all) and np.array_equal(grad.numpy(), g_all))
    finally:
        dist.destroy_process_group()


def test_gather_sharded_world2():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] and out[1]

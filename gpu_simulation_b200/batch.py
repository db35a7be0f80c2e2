"""Batched ring-Ising circuits: thousands of independent (n, L, h) circuits per
kernel launch (include/rsv.h ``rsv_batch_*``).

The reference evaluates one circuit per ``RingIsingCudaBackend`` object
(``cpp/ising_cuda_backend.hpp:22-49``); a batch there is a Python loop over
backends.  Here one persistent kernel takes the whole list: one CTA per
circuit at a time, circuits handed out longest first from an atomic counter,
every circuit running the pass plan the single-circuit engine would run.

Packed layout: circuit ``c`` owns ``params[off[c] : off[c] + 2*n_c*L_c]`` with
the per-circuit layout ``(L, n, 2)`` flattened; gradients use the same packing.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, load_library

MAX_QUBITS = 16
MAX_LAYERS = 64


def param_offsets(num_qubits, num_layers) -> np.ndarray:
    """Offsets of every circuit's parameters in the packed array (length count+1)."""
    sizes = 2 * np.asarray(num_qubits, dtype=np.int64) * np.asarray(num_layers, dtype=np.int64)
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)


def synthetic_batch(count: int = 4096, seed: int = 7, n_range=(6, 16), layer_range=(1, 16),
                    field_range=(0.2, 2.0)):
    """Seeded batch of random circuits: per circuit, in this order from one
    ``numpy.random.default_rng(seed)``: n ~ U{n_range}, L ~ U{layer_range},
    h ~ U[field_range), angles (L, n, 2) ~ U[0, 2 pi).

    Returns (num_qubits int32[count], num_layers int32[count], fields f64[count],
    packed params f64[sum 2nL]).
    """
    rng = np.random.default_rng(seed)
    ns = np.empty(count, dtype=np.int32)
    ls = np.empty(count, dtype=np.int32)
    hs = np.empty(count, dtype=np.float64)
    chunks = []
    for c in range(count):
        ns[c] = rng.integers(n_range[0], n_range[1] + 1)
        ls[c] = rng.integers(layer_range[0], layer_range[1] + 1)
        hs[c] = rng.uniform(field_range[0], field_range[1])
        chunks.append(rng.uniform(0.0, 2.0 * np.pi, size=(int(ls[c]), int(ns[c]), 2)).reshape(-1))
    params = np.concatenate(chunks) if chunks else np.zeros(0)
    return ns, ls, hs, params


def circuit_cost(num_qubits, num_layers) -> np.ndarray:
    """Relative cost of each circuit (amplitudes x layers), for sharding and ordering."""
    n = np.maximum(np.asarray(num_qubits, dtype=np.int64), 12)
    return (np.int64(1) << n) * np.asarray(num_layers, dtype=np.int64)


def shard_circuits(num_qubits, num_layers, world_size: int) -> list[np.ndarray]:
    """Split circuit indices into ``world_size`` contiguous ranges of nearly
    equal total cost (circuits are independent, so no data-path collective is
    needed; each rank evaluates its range and the results are gathered)."""
    cost = circuit_cost(num_qubits, num_layers).astype(np.float64)
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world_size):
        bounds.append(int(np.searchsorted(cum, total * r / world_size, side="left")))
    bounds.append(len(cost))
    bounds = np.maximum.accumulate(np.asarray(bounds))
    return [np.arange(bounds[r], bounds[r + 1]) for r in range(world_size)]


def gather_sharded(local_energy, local_grad, shards, offsets, group=None):
    """All-gather every rank's results for its shard (``shard_circuits``) into
    the full energies [count] and packed gradients [num_params], in circuit
    order.  Shards are contiguous ranges in rank order, so the gathered pieces
    only need their padding trimmed.  Works on any torch.distributed backend
    whose device holds the tensors (NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    counts = [len(s) for s in shards]
    sizes = [int(offsets[s[-1] + 1] - offsets[s[0]]) if len(s) else 0 for s in shards]
    pad_e, pad_g = max(1, max(counts)), max(1, max(sizes))
    dev = local_energy.device

    def padded(x, n):
        out = torch.zeros(n, dtype=torch.float64, device=dev)
        out[: x.numel()] = x
        return out

    e_parts = [torch.empty(pad_e, dtype=torch.float64, device=dev) for _ in range(world)]
    g_parts = [torch.empty(pad_g, dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(e_parts, padded(local_energy, pad_e), group=group)
    dist.all_gather(g_parts, padded(local_grad, pad_g), group=group)
    energy = torch.cat([e_parts[r][: counts[r]] for r in range(world)])
    grad = torch.cat([g_parts[r][: sizes[r]] for r in range(world)])
    return energy, grad


class BatchEngine:
    """Owns one ``rsv_batch`` (scratch for ``slots`` circuits in flight on the current GPU)."""

    def __init__(self, max_qubits: int = MAX_QUBITS, slots: int = 0) -> None:
        self._lib = load_library()
        h = ctypes.c_void_p()
        check(self._lib.rsv_batch_create(int(max_qubits), int(slots), ctypes.byref(h)))
        self._h = h
        self.max_qubits = int(max_qubits)
        self.count = 0
        self.num_params = 0
        self.offsets = np.zeros(1, dtype=np.int64)
        self.max_slots = self.slots

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rsv_batch_destroy(self._h)
            self._h = None

    def __del__(self) -> None:  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _arrays(num_qubits, num_layers, fields):
        ns = np.ascontiguousarray(np.asarray(num_qubits, dtype=np.int32).reshape(-1))
        ls = np.ascontiguousarray(np.asarray(num_layers, dtype=np.int32).reshape(-1))
        hs = np.ascontiguousarray(np.asarray(fields, dtype=np.float64).reshape(-1))
        if not (ns.size == ls.size == hs.size):
            raise ValueError("num_qubits, num_layers and fields must have the same length")
        return ns, ls, hs

    def set_circuits(self, num_qubits, num_layers, fields) -> np.ndarray:
        """Describe the circuits of the following runs; returns the packed offsets."""
        ns, ls, hs = self._arrays(num_qubits, num_layers, fields)
        check(self._lib.rsv_batch_set_circuits(self._h, ns.size, ns.ctypes.data, ls.ctypes.data,
                                               hs.ctypes.data))
        self.count = int(ns.size)
        self.offsets = param_offsets(ns, ls)
        self.num_params = int(self.offsets[-1])
        return self.offsets

    @property
    def slots(self) -> int:
        v = ctypes.c_int()
        check(self._lib.rsv_batch_info(self._h, None, None, ctypes.byref(v), None))
        return int(v.value)

    def set_active_slots(self, slots: int) -> None:
        check(self._lib.rsv_batch_set_active_slots(self._h, int(slots)))

    def set_cluster(self, cluster: int) -> None:
        """CTAs per thread-block cluster (1, 2, 4 or 8): a large circuit is
        spread over up to this many SMs, and the cluster's CTAs add their
        sums through distributed shared memory."""
        check(self._lib.rsv_batch_set_cluster(self._h, int(cluster)))

    def cluster(self) -> dict:
        c, g, m = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.rsv_batch_cluster(self._h, ctypes.byref(c), ctypes.byref(g), ctypes.byref(m)))
        return {"cluster": c.value, "groups": g.value, "max_active_clusters": m.value}

    def device_bytes(self) -> int:
        v = ctypes.c_size_t()
        check(self._lib.rsv_batch_info(self._h, None, None, None, ctypes.byref(v)))
        return int(v.value)

    def run_device(self, params, energy_out, grad_out=None, stream=None) -> None:
        """Enqueue the batch on CUDA tensors (float64, contiguous): params and
        grad_out [num_params], energy_out [count].  Runs on ``stream`` or the
        current torch stream; capturable into a CUDA graph."""
        import torch

        for t in (params, energy_out) + ((grad_out,) if grad_out is not None else ()):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("device tensors must be contiguous float64 CUDA tensors")
        if params.numel() != self.num_params:
            raise ValueError(f"params has {params.numel()} values, the circuits need {self.num_params}")
        if energy_out.numel() < self.count:
            raise ValueError("energy_out is shorter than the circuit count")
        if grad_out is not None and grad_out.numel() != self.num_params:
            raise ValueError("grad_out does not match the circuits")
        s = stream if stream is not None else torch.cuda.current_stream(params.device)
        check(self._lib.rsv_batch_run_device(
            self._h, params.data_ptr(), energy_out.data_ptr(),
            grad_out.data_ptr() if grad_out is not None else None, s.cuda_stream))

    def energy_and_grad(self, num_qubits, num_layers, fields, params, compute_gradient: bool = True):
        """Host arrays in and out (synchronous): (energies f64[count], packed gradient or None)."""
        ns, ls, hs = self._arrays(num_qubits, num_layers, fields)
        flat = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        e = np.empty(ns.size, dtype=np.float64)
        g = np.empty(flat.size, dtype=np.float64) if compute_gradient else None
        check(self._lib.rsv_batch_energy_and_grad(
            self._h, ns.size, ns.ctypes.data, ls.ctypes.data, hs.ctypes.data, flat.ctypes.data,
            flat.size, e.ctypes.data, g.ctypes.data if g is not None else None, None))
        self.count = int(ns.size)
        self.offsets = param_offsets(ns, ls)
        self.num_params = int(self.offsets[-1])
        return e, g

    def capture_graph(self, params, energy_out, grad_out=None):
        """CUDA graph of one batch run on these tensors (replay with ``.replay()``)."""
        import torch

        s = torch.cuda.Stream(device=params.device)
        s.wait_stream(torch.cuda.current_stream(params.device))
        with torch.cuda.stream(s):
            self.run_device(params, energy_out, grad_out, stream=s)  # warm-up outside capture
        torch.cuda.current_stream(params.device).wait_stream(s)
        torch.cuda.synchronize(params.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.run_device(params, energy_out, grad_out)
        return graph

    def autotune(self, params, energy_out, grad_out=None, candidates=None, repeats: int = 3) -> dict:
        """Time the batch for each cluster size (1, 2, 4, 8 CTAs) and a few
        numbers of CTAs in flight, and keep the fastest (bigger clusters spread
        large circuits over more SMs and keep fewer of them, and their states,
        in flight; more CTAs keep every SM busy).  Returns
        {"cluster x CTAs": ms} and sets the best."""
        import torch

        full = self.max_slots
        if candidates is None:
            candidates = []
            for c in (1, 2, 4, 8):
                if c > full:
                    continue
                for k in sorted({max(c, (full * f // 4) // c * c) for f in (2, 3, 4)}):
                    candidates.append((c, k))
        times = {}
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        for c, k in candidates:
            try:
                self.set_cluster(c)
            except ValueError:
                continue  # no cluster of this size fits
            self.set_active_slots(k)
            self.run_device(params, energy_out, grad_out)
            a.record()
            for _ in range(repeats):
                self.run_device(params, energy_out, grad_out)
            b.record()
            b.synchronize()
            times[(c, int(k))] = a.elapsed_time(b) / repeats
        best = min(times, key=times.get)
        self.set_cluster(best[0])
        self.set_active_slots(best[1])
        return {f"{c}x{k}": ms for (c, k), ms in times.items()}

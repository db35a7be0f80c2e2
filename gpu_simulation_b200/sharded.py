"""Sharded single circuit: one ring-Ising circuit split over N = 2^g GPUs.

For circuits whose state does not fit one GPU (n >= 33: one complex128 state
vector of 2^33 amplitudes is 128 GiB; the engine keeps four per rank).  The
reference runs every n on one device and has no multi-GPU path
(cpp/ising_cuda_backend.cu:229-241); the results are the same energy and
gradient as its ``structured_adjoint`` strategy (layout
``(l*n + w)*2 + {0: theta, 1: phi}``).

Each rank holds 2^(n-g) amplitudes in one of two layouts of the global index
(include/rsv_shard.h): C, where wires 0..n-g-1 are local, and S, where wires
0..n-2g-1 and n-g..n-1 are.  One layer forward:

  1. ``rotate_local``: the gates of wires 0..n-g-1 (local in C), own tile
     kernels, in tangent form: (1/f) diag(1, e^{i phi}) RY(theta), the
     layer's prod f restored in step 3;
  2. C -> S: one all-to-all of 2^(n-2g)-amplitude blocks, no packing;
  3. ``ring_pack``: the gates of wires n-g..n-1 (local in S) fused with the sort of
     every amplitude by the rank that owns its image under the CNOT ring;
  4. all-to-all, then ``ring_unpack``: the state after the ring, in C.

The energy takes the X terms of wires 0..n-g-1 in C, and those of wires
n-g..n-1 on the way back to S at the start of the backward (they are local
there in the pre-ring frame).  The backward runs the same exchanges in reverse
on psi and lambda with the gradient sums of the reference's inverse walk.  So
a layer costs two all-to-alls of one vector forward and of two vectors
backward; the energy and gradient are one all-gather of 2 + 2nL doubles,
summed in rank order (deterministic).

Ranks are either the processes of a ``torch.distributed`` group (NCCL, one
GPU each: ``group=``) or ``virtual_ranks=N`` shards held by this process on
one device, whose all-to-alls are device copies (the same kernels and the same
exchange schedule; used to check the sharded path on one GPU).
"""

from __future__ import annotations

import numpy as np

from ._lib import check, load_library


class CudaShardOps:
    """The per-rank kernels of include/rsv_shard.h on CUDA tensors (librsv.so).

    Every call is asynchronous on the current torch stream of the tensors'
    device.  There is no CPU implementation: the library must be built and the
    tensors must be CUDA tensors.
    """

    def __init__(self) -> None:
        self._lib = load_library()

    @staticmethod
    def _stream(t):
        import torch

        if not t.is_cuda:
            raise ValueError("the sharded engine's kernels need CUDA tensors")
        return ctypes_stream(torch.cuda.current_stream(t.device))

    def check(self, n: int, g: int) -> None:
        check(self._lib.rsv_shard_check(int(n), int(g)))

    def scratch_doubles(self, n: int, g: int) -> int:
        return int(self._lib.rsv_shard_scratch_doubles(int(n), int(g)))

    def coef(self, n, L, params, coef):
        check(self._lib.rsv_shard_coef(n, L, params.data_ptr(), coef.data_ptr(), self._stream(params)))

    def init(self, n, g, rank, psi):
        check(self._lib.rsv_shard_init(n, g, rank, psi.data_ptr(), self._stream(psi)))

    def rotate_local(self, n, g, layer, coef, psi):
        check(self._lib.rsv_shard_rotate_local(n, g, layer, coef.data_ptr(), psi.data_ptr(), self._stream(psi)))

    def rotate_local_adjoint(self, n, g, L, layer, coef, psi, lam, scratch, result):
        check(self._lib.rsv_shard_rotate_local_adjoint(n, g, L, layer, coef.data_ptr(), psi.data_ptr(),
                                                       lam.data_ptr(), scratch.data_ptr(), result.data_ptr(),
                                                       self._stream(psi)))

    def energy_local(self, n, g, rank, field, psi, lam, scratch, result):
        check(self._lib.rsv_shard_energy_local(n, g, rank, float(field), psi.data_ptr(), lam.data_ptr(),
                                               scratch.data_ptr(), result.data_ptr(), self._stream(psi)))

    def ring_pack(self, n, g, rank, layer, coef, psi_s, send):
        check(self._lib.rsv_shard_ring_pack(n, g, rank, layer, coef.data_ptr(), psi_s.data_ptr(), send.data_ptr(),
                                            self._stream(psi_s)))

    def ring_unpack(self, n, g, rank, recv, psi_c):
        check(self._lib.rsv_shard_ring_unpack(n, g, rank, recv.data_ptr(), psi_c.data_ptr(), self._stream(recv)))

    def ring_pack_adjoint(self, n, g, rank, psi_c, lam_c, send_psi, send_lam):
        check(self._lib.rsv_shard_ring_pack_adjoint(n, g, rank, psi_c.data_ptr(), lam_c.data_ptr(),
                                                    send_psi.data_ptr(), send_lam.data_ptr(), self._stream(psi_c)))

    def ring_unpack_adjoint(self, n, g, rank, L, layer, coef, field, add_field, recv_psi, recv_lam, psi_s, lam_s,
                            scratch, result):
        check(self._lib.rsv_shard_ring_unpack_adjoint(
            n, g, rank, L, layer, coef.data_ptr() if coef is not None else None, float(field), int(bool(add_field)),
            recv_psi.data_ptr(), recv_lam.data_ptr(), psi_s.data_ptr(), lam_s.data_ptr(), scratch.data_ptr(),
            result.data_ptr(), self._stream(psi_s)))


def ctypes_stream(stream) -> int:
    """cudaStream_t of a torch.cuda.Stream as an integer for ctypes."""
    return int(stream.cuda_stream)


class _Shard:
    """One rank's buffers: psi and lambda, each with an exchange partner."""

    def __init__(self, torch, rank: int, local: int, num_results: int, scratch: int, coef: int, device) -> None:
        self.rank = rank
        cplx = dict(dtype=torch.complex128, device=device)
        self.psi = torch.zeros(local, **cplx)
        self.psi_alt = torch.zeros(local, **cplx)
        self.lam = torch.zeros(local, **cplx)
        self.lam_alt = torch.zeros(local, **cplx)
        self.scratch = torch.zeros(max(1, scratch), dtype=torch.float64, device=device)
        self.result = torch.zeros(num_results, dtype=torch.float64, device=device)
        self.coef = torch.zeros(4 * coef, dtype=torch.float64, device=device)
        self.params = torch.zeros(2 * coef, dtype=torch.float64, device=device)

    def swap_psi(self) -> None:
        self.psi, self.psi_alt = self.psi_alt, self.psi

    def swap_lam(self) -> None:
        self.lam, self.lam_alt = self.lam_alt, self.lam


class ShardedEngine:
    """Energy and gradient of one circuit whose state is split over 2^g ranks.

    ``group``: a ``torch.distributed`` process group (NCCL), one rank and one
    GPU per process, its size a power of two up to 8; the tensors live on
    ``device`` (default: the current CUDA device).  ``virtual_ranks``: N shards
    held by this process on ``device`` instead.  ``ops``: the per-rank kernels
    (default: ``CudaShardOps``, the library's CUDA kernels).
    """

    def __init__(self, num_qubits: int, num_layers: int, field: float = 1.0, *, group=None,
                 virtual_ranks: int | None = None, device=None, ops=None) -> None:
        import torch

        self._torch = torch
        if (group is None) == (virtual_ranks is None):
            raise ValueError("give exactly one of group (torch.distributed) or virtual_ranks")
        self.group = group
        if group is not None:
            import torch.distributed as dist

            self._dist = dist
            self.world = dist.get_world_size(group)
            self.local_ranks = [dist.get_rank(group)]
        else:
            self._dist = None
            self.world = int(virtual_ranks)
            self.local_ranks = list(range(self.world))
        if self.world < 1 or self.world & (self.world - 1):
            raise ValueError("the number of ranks must be a power of two")
        self.g = self.world.bit_length() - 1
        self.n = int(num_qubits)
        self.L = int(num_layers)
        self.field = float(field)
        self.num_params = 2 * self.n * self.L
        self.ops = ops if ops is not None else CudaShardOps()
        self.ops.check(self.n, self.g)
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.local_size = 1 << (self.n - self.g)
        self.block = 1 << (self.n - 2 * self.g)
        scratch = self.ops.scratch_doubles(self.n, self.g)
        self.shards = [_Shard(torch, r, self.local_size, 2 + self.num_params, scratch, self.n * self.L, self.device)
                       for r in self.local_ranks]

    # ------------------------------------------------------------ exchanges
    def _all_to_all(self, outs, ins) -> None:
        """Block j of every rank's input goes to rank j, at block <sender>."""
        if self._dist is not None:
            self._dist.all_to_all_single(outs[0], ins[0], group=self.group)
            return
        N, B = self.world, self.block
        for dst in range(N):
            ov = outs[dst].view(N, B)
            for src in range(N):
                ov[src].copy_(ins[src].view(N, B)[dst])

    def _sum_results(self):
        """Energy and gradient: the ranks' result vectors added in rank order."""
        torch = self._torch
        if self._dist is not None:
            mine = self.shards[0].result
            parts = [torch.empty_like(mine) for _ in range(self.world)]
            self._dist.all_gather(parts, mine, group=self.group)
        else:
            parts = [s.result for s in self.shards]
        total = parts[0].clone()
        for p in parts[1:]:
            total += p
        return total

    def _swap_layout(self, both: bool) -> None:
        """C <-> S for psi (and lambda)."""
        self._all_to_all([s.psi_alt for s in self.shards], [s.psi for s in self.shards])
        for s in self.shards:
            s.swap_psi()
        if both:
            self._all_to_all([s.lam_alt for s in self.shards], [s.lam for s in self.shards])
            for s in self.shards:
                s.swap_lam()

    # ------------------------------------------------------------ the circuit
    def _load_params(self, params) -> None:
        torch = self._torch
        if isinstance(params, torch.Tensor):
            flat = params.detach().reshape(-1).to(dtype=torch.float64)
        else:
            flat = torch.from_numpy(np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1)))
        if flat.numel() != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {flat.numel()}")
        for s in self.shards:
            s.params.copy_(flat, non_blocking=False)
            s.result.zero_()
            self.ops.coef(self.n, self.L, s.params, s.coef)

    def _forward(self) -> None:
        n, g, ops = self.n, self.g, self.ops
        for s in self.shards:
            ops.init(n, g, s.rank, s.psi)
        for layer in range(self.L):
            for s in self.shards:
                ops.rotate_local(n, g, layer, s.coef, s.psi)
            self._swap_layout(both=False)
            for s in self.shards:
                ops.ring_pack(n, g, s.rank, layer, s.coef, s.psi, s.psi_alt)
            self._all_to_all([s.psi for s in self.shards], [s.psi_alt for s in self.shards])
            for s in self.shards:
                ops.ring_unpack(n, g, s.rank, s.psi, s.psi_alt)
                s.swap_psi()

    def _ring_back(self, layer: int, add_field: bool) -> None:
        """psi, lambda from C to S through the inverse ring (and the wires n-g..n-1 of `layer`)."""
        n, g, ops = self.n, self.g, self.ops
        for s in self.shards:
            ops.ring_pack_adjoint(n, g, s.rank, s.psi, s.lam, s.psi_alt, s.lam_alt)
        self._all_to_all([s.psi for s in self.shards], [s.psi_alt for s in self.shards])
        self._all_to_all([s.lam for s in self.shards], [s.lam_alt for s in self.shards])
        for s in self.shards:
            ops.ring_unpack_adjoint(n, g, s.rank, self.L, layer, s.coef if layer >= 0 else None, self.field,
                                    add_field, s.psi, s.lam, s.psi_alt, s.lam_alt, s.scratch, s.result)
            s.swap_psi()
            s.swap_lam()

    def energy_and_grad(self, params, compute_gradient: bool = True):
        """(energy, gradient f64[2nL] or None), the same on every rank."""
        if self.device.type == "cuda":
            # the library launches on the current device: make it the shards' device
            with self._torch.cuda.device(self.device):
                return self._energy_and_grad(params, compute_gradient)
        return self._energy_and_grad(params, compute_gradient)

    def _energy_and_grad(self, params, compute_gradient: bool):
        n, g, ops = self.n, self.g, self.ops
        self._load_params(params)
        self._forward()
        for s in self.shards:
            ops.energy_local(n, g, s.rank, self.field, s.psi, s.lam, s.scratch, s.result)
        if not compute_gradient:
            self._ring_back(-1, True)
        else:
            for layer in range(self.L - 1, -1, -1):
                self._ring_back(layer, layer == self.L - 1)
                self._swap_layout(both=True)
                for s in self.shards:
                    ops.rotate_local_adjoint(n, g, self.L, layer, s.coef, s.psi, s.lam, s.scratch, s.result)
        total = self._sum_results().cpu().numpy()
        energy = float(total[0] + total[1])
        return energy, (total[2:].copy() if compute_gradient else None)

    def energy(self, params) -> float:
        return self.energy_and_grad(params, compute_gradient=False)[0]


def _autograd_function():
    import torch

    class ShardedRingIsingEnergy(torch.autograd.Function):
        """Energy of the ring-Ising ansatz through a ``ShardedEngine``, for
        torch optimisers on circuits too large for one GPU.  The adjoint sweep
        yields the energy and the whole gradient in one call, so the forward
        keeps the gradient and the backward only scales it by the incoming
        grad; every rank gets the same energy and gradient."""

        @staticmethod
        def forward(ctx, params, engine):
            energy, grad = engine.energy_and_grad(params.detach())
            ctx.shape = params.shape
            ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype, device=params.device))
            return torch.tensor(energy, dtype=params.dtype, device=params.device)

        @staticmethod
        def backward(ctx, grad_output):
            (grad,) = ctx.saved_tensors
            return (grad * grad_output).reshape(ctx.shape), None

    return ShardedRingIsingEnergy


_SHARDED_FN = None


def sharded_ring_ising_energy(params, engine: ShardedEngine):
    """Differentiable energy (0-d tensor) of params of shape (L, n, 2) or flat,
    evaluated by ``engine`` (a ``ShardedEngine``)."""
    global _SHARDED_FN
    if _SHARDED_FN is None:
        _SHARDED_FN = _autograd_function()
    return _SHARDED_FN.apply(params, engine)

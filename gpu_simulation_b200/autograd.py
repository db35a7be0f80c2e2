"""``torch.autograd.Function`` whose backward is the engine's adjoint sweep.

``RingIsingEnergy.apply(params, engine)`` returns the energy as a 0-d float64
CUDA tensor.  The forward runs the forward sweep and the energy kernel and
keeps the final state and lambda = H psi on the device; ``backward`` then runs
only the adjoint sweep (``rsv_backward_device``) and scales the gradient by the
incoming grad.  If the engine has run another call in between (a second
forward before backward), backward recomputes forward + adjoint from the saved
parameters, so results never mix two forwards.  Everything stays on the GPU;
there is no host round trip and no CPU fallback.
"""

from __future__ import annotations

import ctypes

import torch

from ._lib import RSV_ERR_STALE_STATE, check
from .engine import Engine


class RingIsingEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params: torch.Tensor, engine: Engine) -> torch.Tensor:
        if not params.is_cuda or params.dtype != torch.float64:
            raise ValueError("params must be a float64 CUDA tensor")
        flat = params.detach().reshape(-1).contiguous()
        if flat.numel() != engine.num_params:
            raise ValueError(f"expected {engine.num_params} parameters, got {flat.numel()}")
        energy = torch.empty(1, dtype=torch.float64, device=params.device)
        stream = torch.cuda.current_stream(params.device)
        gen = ctypes.c_ulonglong()
        check(engine._lib.rsv_forward_device(engine._h, flat.data_ptr(), flat.numel(),
                                             energy.data_ptr(), ctypes.byref(gen), stream.cuda_stream))
        ctx.engine = engine
        ctx.generation = gen.value
        ctx.shape = params.shape
        ctx.save_for_backward(flat)
        return energy.reshape(())

    @staticmethod
    def backward(ctx, grad_output: torch.Tensor):
        (flat,) = ctx.saved_tensors
        engine: Engine = ctx.engine
        grad = torch.empty_like(flat)
        stream = torch.cuda.current_stream(flat.device)
        status = engine._lib.rsv_backward_device(engine._h, ctx.generation, grad.data_ptr(),
                                                 stream.cuda_stream)
        if status == RSV_ERR_STALE_STATE:
            # the engine's buffers were reused by another call: recompute
            scratch = torch.empty(1, dtype=torch.float64, device=flat.device)
            engine.energy_and_grad_device(flat, scratch, grad, stream)
        else:
            check(status)  # any other failure is raised, never retried
        return (grad * grad_output).reshape(ctx.shape), None


def ring_ising_energy(params: torch.Tensor, engine: Engine) -> torch.Tensor:
    """Differentiable energy of the ring-Ising ansatz for params of shape (L, n, 2) or flat."""
    return RingIsingEnergy.apply(params, engine)

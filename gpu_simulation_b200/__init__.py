"""B200-native ring-Ising statevector engine (structured adjoint energy + gradient).

Public surface
  * ``Engine``                      C-ABI handle (host and device entry points)
  * ``RingIsingAdjointBackend`` / ``StandaloneBackendConfig``
                                    mirror of the reference's Python wrapper
  * ``ring_ising_energy`` / ``RingIsingEnergy``
                                    torch.autograd.Function (backward = adjoint kernels)
  * ``describe_plan``               launch schedule of one call (host only)
  * ``BatchEngine``                 thousands of independent circuits per kernel launch
  * ``training.run_standalone``     device-resident gradient-descent loop (CUDA-graph steps)
  * ``warmstart``                   learned warm start (FP32 network, own kernels)

The compiled pieces are built in-tree by ``python -m gpu_simulation_b200.build``.
"""

from __future__ import annotations

from .backend import RingIsingAdjointBackend, StandaloneBackendConfig
from .batch import BatchEngine
from .engine import Engine, describe_plan

__all__ = [
    "BatchEngine",
    "Engine",
    "RingIsingAdjointBackend",
    "RingIsingEnergy",
    "StandaloneBackendConfig",
    "describe_plan",
    "ring_ising_energy",
]


def __getattr__(name):
    # torch is imported lazily: the host-only parts work without it.
    if name in ("RingIsingEnergy", "ring_ising_energy"):
        from . import autograd

        return getattr(autograd, name)
    raise AttributeError(name)

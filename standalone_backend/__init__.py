"""Drop-in extension package for the reference's ``standalone_backend``.

``standalone_backend._cuda_backend`` is the B200 (sm_100a) build of the
ring-Ising structured-adjoint engine with the reference's pybind11 API
(class ``RingIsingCudaBackend``, module function ``energy_and_grad``).
Build it with ``python -m gpu_simulation_b200.build``.
"""

from __future__ import annotations

__all__ = ["_cuda_backend"]

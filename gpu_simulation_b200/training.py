"""Device-resident VQE training loop (the reference's standalone workflow).

The reference's ``run_standalone`` (ring_ising/workflows/standalone.py:90-167)
runs ``run_gradient_descent_loop`` (ring_ising/training/loop.py:75-130): per
step one ``energy_and_grad`` of the current angles and a plain update
``params - stepsize * grad`` (ring_ising/workflows/common.py:23-25), with the
angles round-tripping through the host every step.  Here the angles, the
gradient and the per-step metrics stay on the GPU: one step is the engine's
device entry point plus one fused update kernel (``rsv_gd_step_f64``), and the
step can be captured once into a CUDA graph and replayed ``steps`` times.  The
host reads the histories once at the end.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from ._lib import check, load_library
from .engine import Engine


def make_initial_params(num_qubits: int, layers: int, seed: int, init_scale: float) -> np.ndarray:
    """Seeded initial angles, shape (layers, num_qubits, 2): init_scale * N(0, 1)
    from default_rng(seed) (reference ring_ising/params.py:8-20)."""
    rng = np.random.default_rng(seed)
    return np.asarray(init_scale * rng.standard_normal((layers, num_qubits, 2)), dtype=np.float64)


@dataclass(frozen=True)
class StepMetric:
    """Per-step metrics (reference ring_ising/training/loop.py:17-23): the energy
    evaluated at the angles before the step's update, and the gradient norm."""

    step: int
    energy: float
    grad_norm: float
    step_wall_s: float


@dataclass
class TrainingRunResult:
    """Outputs of one run (reference ring_ising/training/result.py:18-27)."""

    backend_label: str
    final_params: np.ndarray
    final_energy: float
    step_metrics: tuple[StepMetric, ...]
    wall_s: float
    metadata: dict[str, Any] = field(default_factory=dict)


def run_gradient_descent_device(engine: Engine, params, steps: int, stepsize: float,
                                use_graph: bool = True) -> TrainingRunResult:
    """Plain gradient descent with the angles resident on the GPU.

    Every step evaluates the energy and gradient of the current angles and
    applies ``params - stepsize * grad``; the step energies and gradient norms
    are recorded on the device.  With ``use_graph`` one step is captured into
    a CUDA graph and replayed.  Per-step wall time is the loop's GPU time
    divided evenly (the steps are not synchronised individually).
    """
    import torch

    if steps < 1:
        raise ValueError("steps must be at least 1.")
    lib = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.as_tensor(np.asarray(params, dtype=np.float64).reshape(-1)).to(dev).contiguous()
    if p.numel() != engine.num_params:
        raise ValueError("num_params does not match the circuit.")
    g = torch.empty_like(p)
    e = torch.empty(1, dtype=torch.float64, device=dev)
    e_hist = torch.empty(steps, dtype=torch.float64, device=dev)
    n_hist = torch.empty(steps, dtype=torch.float64, device=dev)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)

    def step(stream):
        engine.energy_and_grad_device(p, e, g, stream=stream)
        check(lib.rsv_gd_step_f64(p.data_ptr(), g.data_ptr(), p.numel(), float(stepsize), e.data_ptr(),
                                  e_hist.data_ptr(), n_hist.data_ptr(), counter.data_ptr(), stream.cuda_stream))

    # one evaluation outside the timed loop and the capture configures every
    # kernel once (the angles are not updated by it)
    engine.energy_and_grad_device(p, e, g)
    torch.cuda.synchronize(dev)
    start = time.perf_counter()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    if use_graph:
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.graph(graph, stream=side):
            step(side)
        # capture records the launches without running them
        a.record()
        for _ in range(steps):
            graph.replay()
        b.record()
    else:
        s = torch.cuda.current_stream(dev)
        a.record()
        for _ in range(steps):
            step(s)
        b.record()
    b.synchronize()
    gpu_ms = a.elapsed_time(b)
    if int(counter.item()) != steps:
        raise RuntimeError(f"step counter {int(counter.item())} != {steps}")
    final_params = p.cpu().numpy().reshape(engine.num_layers, engine.num_qubits, 2)
    final_energy = engine.energy(final_params)
    energies = e_hist.cpu().numpy()
    norms = n_hist.cpu().numpy()
    per = gpu_ms * 1e-3 / steps
    metrics = tuple(StepMetric(step=k + 1, energy=float(energies[k]), grad_norm=float(norms[k]),
                               step_wall_s=per) for k in range(steps))
    return TrainingRunResult(
        backend_label="standalone_b200",
        final_params=final_params,
        final_energy=float(final_energy),
        step_metrics=metrics,
        wall_s=time.perf_counter() - start,
        metadata={"gpu_ms": gpu_ms, "cuda_graph": bool(use_graph),
                  "gradient_strategy": "structured_adjoint"},
    )


def run_adam_device(engine: Engine, params, steps: int, lr: float = 0.05, betas=(0.9, 0.999),
                    eps: float = 1e-8, use_graph: bool = True) -> dict:
    """``steps`` Adam steps with the angles resident on the GPU, the update of
    ``torch.optim.Adam`` (bias-corrected, no weight decay) applied by one fused
    kernel (``rsv_adam_vqe_step_f64``): the same trajectory as a torch Adam loop
    over the autograd Function, without the per-step Python and optimiser
    launches.  With ``use_graph`` one (energy_and_grad, Adam) step is captured
    into a CUDA graph and replayed.  Returns the final angles (flat), the
    energy evaluated at the start of every step, and the GPU time of the loop.
    """
    import torch

    if steps < 1:
        raise ValueError("steps must be at least 1.")
    lib = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.as_tensor(np.asarray(params, dtype=np.float64).reshape(-1)).to(dev).contiguous()
    if p.numel() != engine.num_params:
        raise ValueError("num_params does not match the circuit.")
    g = torch.empty_like(p)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    e = torch.empty(1, dtype=torch.float64, device=dev)
    e_hist = torch.empty(steps, dtype=torch.float64, device=dev)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    b1, b2 = float(betas[0]), float(betas[1])

    def step(stream):
        engine.energy_and_grad_device(p, e, g, stream=stream)
        check(lib.rsv_adam_vqe_step_f64(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(),
                                        float(lr), b1, b2, float(eps), e.data_ptr(), e_hist.data_ptr(),
                                        counter.data_ptr(), stream.cuda_stream))

    # one evaluation outside the timed loop configures every kernel once
    engine.energy_and_grad_device(p, e, g)
    torch.cuda.synchronize(dev)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    graph = None
    if use_graph:
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.graph(graph, stream=side):
            step(side)
        # capture records the launches without running them
        a.record()
        for _ in range(steps):
            graph.replay()
        b.record()
    else:
        s = torch.cuda.current_stream(dev)
        a.record()
        for _ in range(steps):
            step(s)
        b.record()
    b.synchronize()
    gpu_ms = a.elapsed_time(b)
    if int(counter.item()) != steps:
        raise RuntimeError(f"step counter {int(counter.item())} != {steps}")
    out = {"params": p.cpu().numpy(), "energies": e_hist.cpu().numpy(), "gpu_ms": gpu_ms,
           "cuda_graph": bool(use_graph)}
    del graph
    return out


def run_standalone(num_qubits: int, layers: int, steps: int, stepsize: float, field: float = 1.0,
                   seed: int = 7, init_scale: float = 0.3, use_graph: bool = True) -> TrainingRunResult:
    """The reference's standalone workflow on this engine: seeded initial angles,
    ``steps`` plain gradient-descent steps, final energy."""
    engine = Engine(num_qubits, layers, field)
    try:
        params = make_initial_params(num_qubits, layers, seed, init_scale)
        return run_gradient_descent_device(engine, params, steps, stepsize, use_graph=use_graph)
    finally:
        engine.close()

"""Learned warm start for the ring-Ising VQE.

A small fully connected network (FP32, GELU, widths 3 -> 256 -> 256 -> 192
for n = 16, L = 6) maps circuit descriptors (h, n, L) to initial angles.  It is
trained on the converged angles that the plain VQE itself produces across an
h sweep, and it is used only as a warm start: the plain VQE from seeded random
angles stays the fallback, and every reported energy comes from the
simulator.  The reference has no learned part; its VQE loop starts from seeded
random angles (ring_ising/runner.py) and runs plain gradient descent
(ring_ising/optimizers.py).

Everything on the GPU runs through this project's kernels (include/rsv.h):
the batched circuit kernel for the VQE energies and gradients, the FP32
network kernels for training and inference, and fused Adam kernels for both.
Torch only allocates device memory and provides the stream.
"""

from __future__ import annotations

import time

import numpy as np

from ._lib import check, load_library
from .batch import BatchEngine

WIDTHS = (3, 256, 256, 192)


def features(fields, num_qubits, num_layers) -> np.ndarray:
    """Network inputs (h, n / 16, L / 16) as float32 rows."""
    h = np.asarray(fields, dtype=np.float64).reshape(-1)
    n = np.broadcast_to(np.asarray(num_qubits, dtype=np.float64), h.shape)
    L = np.broadcast_to(np.asarray(num_layers, dtype=np.float64), h.shape)
    return np.stack([h, n / 16.0, L / 16.0], axis=1).astype(np.float32)


def unwrap_labels(angles, fields):
    """Choose the 2 pi branch of every converged angle so that each angle
    varies continuously along the h sweep where it can.

    The energy is 2 pi-periodic in every angle (RY(t + 2 pi) = -RY(t), a
    global sign), so converged angles are defined modulo 2 pi only.  Rows are
    unwrapped in order of increasing h (a jump above pi between neighbours
    is taken as a branch change), then every column is shifted by a multiple
    of 2 pi to bring its mean into [-pi, pi].  Returns the relabelled angles
    in the input row order.
    """
    a = np.asarray(angles, dtype=np.float64)
    order = np.argsort(np.asarray(fields, dtype=np.float64).reshape(-1), kind="stable")
    out = np.empty_like(a)
    out[order] = np.unwrap(a[order], axis=0)
    out -= 2.0 * np.pi * np.round(out.mean(axis=0) / (2.0 * np.pi))
    return out


def steps_to_reach(history, target, rel: float = 1e-3) -> np.ndarray:
    """First step s with E_s - target <= rel * |target| per circuit (-1 if never).

    history[s, c] is the energy of circuit c after s optimiser steps.
    """
    hist = np.asarray(history, dtype=np.float64)
    tgt = np.asarray(target, dtype=np.float64)
    ok = hist - tgt[None, :] <= rel * np.abs(tgt)[None, :]
    first = np.argmax(ok, axis=0)
    return np.where(ok.any(axis=0), first, -1)


def init_weights(widths=WIDTHS, seed: int = 0) -> np.ndarray:
    """Packed float32 weights: W ~ N(0, 2 / fan_in) (He), b = 0."""
    rng = np.random.default_rng(seed)
    parts = []
    for l in range(1, len(widths)):
        k, n = widths[l - 1], widths[l]
        parts.append(rng.standard_normal(n * k) * np.sqrt(2.0 / k))
        parts.append(np.zeros(n))
    return np.concatenate(parts).astype(np.float32)


def random_init(count: int, num_qubits: int, num_layers: int, seed: int) -> np.ndarray:
    """Seeded random starting angles U[0, 2 pi), packed (count x L x n x 2)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 2.0 * np.pi, size=count * num_layers * num_qubits * 2)


class WarmStartMLP:
    """The network's weights on the GPU and its training / inference loops."""

    def __init__(self, widths=WIDTHS, seed: int = 0, device=None) -> None:
        import torch

        self._lib = load_library()
        self.widths = tuple(int(w) for w in widths)
        self._w_arr = np.asarray(self.widths, dtype=np.int32)
        self.num_layers = len(self.widths) - 1
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else device
        n_w = self._lib.rsv_mlp_num_weights(self.num_layers, self._w_arr.ctypes.data)
        self.weights = torch.from_numpy(init_weights(self.widths, seed)).to(self.device)
        assert self.weights.numel() == n_w

    def _stream(self):
        import torch

        return torch.cuda.current_stream(self.device).cuda_stream

    def _work(self, batch: int):
        import torch

        nw = self._lib.rsv_mlp_work_floats(self.num_layers, self._w_arr.ctypes.data, batch)
        return torch.empty(max(1, nw), dtype=torch.float32, device=self.device)

    def forward(self, x, work=None):
        """Outputs (batch x widths[-1]) for float32 inputs (batch x widths[0])."""
        import torch

        x = x.to(self.device, torch.float32).contiguous()
        out = torch.empty((x.shape[0], self.widths[-1]), dtype=torch.float32, device=self.device)
        work = self._work(x.shape[0]) if work is None else work
        check(self._lib.rsv_mlp_forward(self.num_layers, self._w_arr.ctypes.data, self.weights.data_ptr(),
                                        x.shape[0], x.data_ptr(), out.data_ptr(), work.data_ptr(),
                                        self._stream()))
        return out

    def gradient(self, x, target):
        """(loss tensor [1], packed weight gradient) of the mean squared error."""
        import torch

        x = x.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        work = self._work(x.shape[0])
        out = self.forward(x, work)
        dout = torch.empty_like(out)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        partials = torch.empty(256, dtype=torch.float32, device=self.device)
        s = self._stream()
        check(self._lib.rsv_mlp_mse(out.numel(), out.data_ptr(), target.data_ptr(), dout.data_ptr(),
                                    loss.data_ptr(), partials.data_ptr(), s))
        grad = torch.empty_like(self.weights)
        ns = self._lib.rsv_mlp_scratch_floats(self.num_layers, self._w_arr.ctypes.data, x.shape[0])
        scratch = torch.empty(max(1, ns), dtype=torch.float32, device=self.device)
        check(self._lib.rsv_mlp_backward(self.num_layers, self._w_arr.ctypes.data, self.weights.data_ptr(),
                                         x.shape[0], x.data_ptr(), work.data_ptr(), dout.data_ptr(),
                                         grad.data_ptr(), scratch.data_ptr(), s))
        return loss, grad

    def train(self, x, target, steps: int = 3000, lr: float = 1e-3, beta1: float = 0.9,
              beta2: float = 0.999, eps: float = 1e-8) -> list[float]:
        """Full-batch Adam on the mean squared error; returns the loss history."""
        import torch

        x = x.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        batch = x.shape[0]
        work = self._work(batch)
        out = torch.empty((batch, self.widths[-1]), dtype=torch.float32, device=self.device)
        dout = torch.empty_like(out)
        ns = self._lib.rsv_mlp_scratch_floats(self.num_layers, self._w_arr.ctypes.data, batch)
        scratch = torch.empty(max(1, ns), dtype=torch.float32, device=self.device)
        grad = torch.empty_like(self.weights)
        m = torch.zeros_like(self.weights)
        v = torch.zeros_like(self.weights)
        losses = torch.empty(steps, dtype=torch.float32, device=self.device)
        partials = torch.empty(256, dtype=torch.float32, device=self.device)
        s = self._stream()
        wa = self._w_arr.ctypes.data
        lib = self._lib
        for step in range(1, steps + 1):
            check(lib.rsv_mlp_forward(self.num_layers, wa, self.weights.data_ptr(), batch, x.data_ptr(),
                                      out.data_ptr(), work.data_ptr(), s))
            check(lib.rsv_mlp_mse(out.numel(), out.data_ptr(), target.data_ptr(), dout.data_ptr(),
                                  losses[step - 1:].data_ptr(), partials.data_ptr(), s))
            check(lib.rsv_mlp_backward(self.num_layers, wa, self.weights.data_ptr(), batch, x.data_ptr(),
                                       work.data_ptr(), dout.data_ptr(), grad.data_ptr(),
                                       scratch.data_ptr(), s))
            check(lib.rsv_adam_f32(self.weights.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(),
                                   self.weights.numel(), lr, beta1, beta2, eps, step, s))
        return losses.cpu().tolist()

    def predict(self, fields, num_qubits: int, num_layers: int) -> np.ndarray:
        """Initial angles, packed float64 (count x L x n x 2)."""
        out = self.forward(__import__("torch").from_numpy(features(fields, num_qubits, num_layers)))
        return out.double().cpu().numpy().reshape(-1)


def vqe_adam(engine: BatchEngine, num_qubits, num_layers, fields, init_params, steps: int,
             lr: float = 0.05, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
    """Plain VQE with Adam on every circuit of a batch at once.

    Each step evaluates all energies and gradients with one batched kernel
    launch, then one fused Adam step updates every angle.  Returns (final
    packed angles f64, history f64[steps + 1, count] with history[s] the
    energies after s steps, GPU milliseconds of the loop).
    """
    import torch

    lib = load_library()
    dev = torch.device("cuda", torch.cuda.current_device())
    engine.set_circuits(num_qubits, num_layers, fields)
    p = torch.as_tensor(np.asarray(init_params, dtype=np.float64)).to(dev).contiguous()
    if p.numel() != engine.num_params:
        raise ValueError("init_params does not match the circuits")
    g = torch.empty_like(p)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    hist = torch.empty((steps + 1, engine.count), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for step in range(1, steps + 1):
        engine.run_device(p, hist[step - 1], g)
        check(lib.rsv_adam_f64(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(), lr,
                               beta1, beta2, eps, step, s))
    engine.run_device(p, hist[steps], None)
    b.record()
    b.synchronize()
    return p.cpu().numpy(), hist.cpu().numpy(), a.elapsed_time(b)


def warm_start_experiment(num_qubits: int = 16, num_layers: int = 6, train_count: int = 512,
                          test_count: int = 128, train_seed: int = 7, test_seed: int = 8,
                          init_seed: int = 1234, vqe_steps: int = 300, vqe_lr: float = 0.05,
                          mlp_schedule=((4000, 3e-3), (4000, 1e-3), (4000, 3e-4)), rel: float = 1e-3,
                          field_range=(0.2, 2.0), engine: BatchEngine | None = None) -> dict:
    """Train the warm-start network on plain-VQE solutions and measure what it gains.

    Train fields: U[field_range) from default_rng(train_seed); held-out
    fields from default_rng(test_seed).  Every circuit's plain VQE starts
    from the same seeded random angles (default_rng(init_seed)).  Returns the
    plain and warm-started steps to reach within ``rel`` (relative) of the
    plain converged energy on the held-out fields, and timings.
    """
    import torch

    eng = engine if engine is not None else BatchEngine(max_qubits=max(num_qubits, 2))
    n, L = int(num_qubits), int(num_layers)
    per = 2 * n * L
    h_train = np.random.default_rng(train_seed).uniform(*field_range, train_count)
    h_test = np.random.default_rng(test_seed).uniform(*field_range, test_count)
    start = random_init(1, n, L, init_seed)

    def run(fields, init):
        k = len(fields)
        return vqe_adam(eng, np.full(k, n), np.full(k, L), fields, init, vqe_steps, vqe_lr)

    t0 = time.perf_counter()
    p_train, hist_train, ms_labels = run(h_train, np.tile(start, train_count))
    labels = unwrap_labels(p_train.reshape(train_count, per), h_train)
    net = WarmStartMLP((3, 256, 256, per) if per != WIDTHS[-1] else WIDTHS)
    x = torch.from_numpy(features(h_train, n, L))
    y = torch.from_numpy(labels.astype(np.float32))
    tm = time.perf_counter()
    losses = []
    for mlp_steps, mlp_lr in mlp_schedule:  # Adam restarted at every learning-rate stage
        losses += net.train(x, y, steps=int(mlp_steps), lr=float(mlp_lr))
    torch.cuda.synchronize()
    mlp_train_s = time.perf_counter() - tm

    _, hist_plain, ms_plain = run(h_test, np.tile(start, test_count))
    e_plain = hist_plain[-1]
    steps_plain = steps_to_reach(hist_plain, e_plain, rel)
    warm = net.predict(h_test, n, L)
    _, hist_warm, ms_warm = run(h_test, warm)
    steps_warm = steps_to_reach(hist_warm, e_plain, rel)
    reached = steps_warm >= 0
    sw = np.where(reached, steps_warm, vqe_steps + 1)
    return {
        "num_qubits": n, "num_layers": L, "train": train_count, "held_out": test_count,
        "vqe_steps": vqe_steps, "rel": rel,
        "mlp_loss_first": float(losses[0]), "mlp_loss_last": float(losses[-1]),
        "mlp_train_s": mlp_train_s, "mlp_steps": int(sum(s for s, _ in mlp_schedule)),
        "label_vqe_ms": ms_labels,
        "plain_steps_median": float(np.median(steps_plain)),
        "plain_steps_mean": float(np.mean(steps_plain)),
        "warm_steps_median": float(np.median(sw)),
        "warm_steps_mean": float(np.mean(sw)),
        "warm_reached_fraction": float(np.mean(reached)),
        "warm_steps_over_plain_median": float(np.median(sw) / max(1.0, np.median(steps_plain))),
        "warm_initial_gap_median": float(np.median((hist_warm[0] - e_plain) / np.abs(e_plain))),
        "plain_initial_gap_median": float(np.median((hist_plain[0] - e_plain) / np.abs(e_plain))),
        "warm_final_minus_plain_median": float(np.median(hist_warm[-1] - e_plain)),
        "plain_vqe_ms": ms_plain, "warm_vqe_ms": ms_warm,
        "ms_per_step_plain": ms_plain / (vqe_steps + 1),
        "plain_ms_to_target_median": float(np.median(steps_plain)) * ms_plain / (vqe_steps + 1),
        "warm_ms_to_target_median": float(np.median(sw)) * ms_warm / (vqe_steps + 1),
        "total_s": time.perf_counter() - t0,
        "steps_plain": steps_plain.tolist(), "steps_warm": steps_warm.tolist(),
    }

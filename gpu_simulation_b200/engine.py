"""Python handle over the C ABI (include/rsv.h): one ``Engine`` per circuit shape.

Host arrays go through ``energy_and_grad`` (synchronous, like the reference's
``RingIsingCudaBackend.energy_and_grad``); CUDA tensors go through
``energy_and_grad_device`` (asynchronous on the current torch stream, no host
round trip).
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, load_library


class Engine:
    """Owns one ``rsv_backend`` (three complex128 state buffers on the current GPU)."""

    def __init__(self, num_qubits: int, num_layers: int, field: float,
                 gradient_strategy: str = "structured_adjoint",
                 structured_rotation_chunk_width: int = 8, double_buffer: bool = False) -> None:
        self._lib = load_library()
        handle = ctypes.c_void_p()
        check(self._lib.rsv_create(int(num_qubits), int(num_layers), float(field),
                                   gradient_strategy.encode(), int(structured_rotation_chunk_width),
                                   int(bool(double_buffer)), ctypes.byref(handle)))
        self._h = handle
        self.num_qubits = int(num_qubits)
        self.num_layers = int(num_layers)
        self.field = float(field)
        self.num_params = 2 * self.num_qubits * self.num_layers

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rsv_destroy(self._h)
            self._h = None

    def __del__(self) -> None:  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    def _flat(self, params) -> np.ndarray:
        flat = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        return flat

    def energy_and_grad(self, params, compute_gradient: bool = True):
        """(energy, gradient f64[2nL] or None) from host parameters."""
        flat = self._flat(params)
        e = ctypes.c_double()
        g = np.empty(self.num_params, dtype=np.float64) if compute_gradient else None
        check(self._lib.rsv_energy_and_grad(
            self._h, flat.ctypes.data, flat.size, int(compute_gradient), ctypes.byref(e),
            g.ctypes.data if g is not None else None, None))
        return float(e.value), g

    def energy(self, params) -> float:
        return self.energy_and_grad(params, compute_gradient=False)[0]

    def profile_energy_and_grad(self, params, compute_gradient: bool = True) -> dict:
        flat = self._flat(params)
        nst = self._lib.rsv_num_stages()
        st = np.zeros(nst, dtype=np.float64)
        e = ctypes.c_double()
        g = np.empty(self.num_params, dtype=np.float64)
        check(self._lib.rsv_profile_energy_and_grad(
            self._h, flat.ctypes.data, flat.size, int(compute_gradient), ctypes.byref(e),
            g.ctypes.data, st.ctypes.data))
        return {
            "energy": float(e.value),
            "gradient": g if compute_gradient else None,
            "timings_ms": {self._lib.rsv_stage_name(i).decode(): float(st[i]) for i in range(nst)},
        }

    def energy_and_grad_device(self, params, energy_out, grad_out=None, stream=None) -> None:
        """Asynchronous call on CUDA tensors (float64, contiguous, on this GPU).

        params: [2nL]; energy_out: [1]; grad_out: [2nL] or None.  Runs on
        ``stream`` (a torch.cuda.Stream) or the current torch stream.
        """
        import torch

        for t in (params, energy_out) + ((grad_out,) if grad_out is not None else ()):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("device tensors must be contiguous float64 CUDA tensors")
        if params.numel() != self.num_params:
            raise ValueError("num_params does not match the circuit.")
        if grad_out is not None and grad_out.numel() != self.num_params:
            raise ValueError("grad_out does not match the circuit.")
        s = stream if stream is not None else torch.cuda.current_stream(params.device)
        check(self._lib.rsv_energy_and_grad_device(
            self._h, params.data_ptr(), params.numel(), energy_out.data_ptr(),
            grad_out.data_ptr() if grad_out is not None else None, s.cuda_stream))

    def benchmark_forward_graph(self, params, repeats: int = 100) -> dict:
        flat = self._flat(params)
        a, b = ctypes.c_double(), ctypes.c_double()
        check(self._lib.rsv_benchmark_forward_graph(self._h, flat.ctypes.data, flat.size, int(repeats),
                                                    ctypes.byref(a), ctypes.byref(b)))
        return {"normal_forward_ms": a.value, "graph_forward_ms": b.value,
                "speedup": a.value / b.value if b.value > 0 else 0.0}

    KINDS = ("tables", "forward_pass", "energy", "backward_pass", "finalize")

    def set_launch_timing(self, enable: bool) -> None:
        """Record CUDA events around every kernel launch of following calls."""
        check(self._lib.rsv_set_launch_timing(self._h, int(bool(enable))))

    def launch_stats(self) -> dict:
        """Per kernel kind: launches, summed ms and summed algorithmic bytes
        recorded since timing was enabled (synchronises, then clears)."""
        k = len(self.KINDS)
        counts = np.zeros(k, dtype=np.int32)
        ms = np.zeros(k, dtype=np.float64)
        by = np.zeros(k, dtype=np.float64)
        check(self._lib.rsv_launch_stats(self._h, counts.ctypes.data, ms.ctypes.data, by.ctypes.data))
        return {name: {"launches": int(counts[i]), "ms": float(ms[i]), "bytes": float(by[i])}
                for i, name in enumerate(self.KINDS)}

    def kernel_launches(self) -> int:
        """Kernels launched by this engine's calls since it was created."""
        out = ctypes.c_ulonglong()
        check(self._lib.rsv_kernel_launches(self._h, ctypes.byref(out)))
        return int(out.value)

    BACKWARD_MODES = {"auto": 0, "uncompute": 1, "checkpoint": 2}

    def set_backward_mode(self, mode: str) -> None:
        """Backward schedule: "uncompute" (three state buffers, psi un-computed
        alongside lambda), "checkpoint" (psi read from forward checkpoints,
        only lambda written) or "auto" (checkpoint while it fits)."""
        if mode not in self.BACKWARD_MODES:
            raise ValueError(f"backward mode must be one of {sorted(self.BACKWARD_MODES)}")
        check(self._lib.rsv_set_backward_mode(self._h, self.BACKWARD_MODES[mode]))

    def backward_mode(self) -> dict:
        m, ck, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.rsv_backward_mode(self._h, ctypes.byref(m), ctypes.byref(ck), ctypes.byref(nb)))
        names = {v: k for k, v in self.BACKWARD_MODES.items()}
        return {"mode": names[m.value], "checkpoint": bool(ck.value), "state_buffers": nb.value}

    def set_analytic_layers(self, max_layers: int) -> None:
        """How many leading layers (0..3, default 3) skip their tile passes:
        the circuit's first layers form a low-bond matrix-product state, written
        in one pass and differentiated from one read of lambda (n >= 13)."""
        check(self._lib.rsv_set_analytic_layers(self._h, int(max_layers)))

    def analytic_layers(self) -> dict:
        m, u = ctypes.c_int(), ctypes.c_int()
        check(self._lib.rsv_analytic_layers(self._h, ctypes.byref(m), ctypes.byref(u)))
        return {"max_layers": m.value, "used": u.value}

    KERNELS_TMA = 1
    KERNELS_FUSED_ENERGY = 2

    def set_kernels(self, tma: bool = True, fused_energy: bool = True) -> None:
        """Backward passes on the TMA-fed kernels where eligible (default) or
        all on the cp.async kernels; with the TMA kernels, fused_energy lets
        the last layer's first backward pass apply the field terms on its
        tile in energy_and_grad calls.  Re-plans the backend."""
        flags = (self.KERNELS_TMA | (self.KERNELS_FUSED_ENERGY if fused_energy else 0)) if tma else 0
        check(self._lib.rsv_set_kernels(self._h, flags))

    def kernels(self) -> dict:
        f, t = ctypes.c_int(), ctypes.c_int()
        check(self._lib.rsv_kernels(self._h, ctypes.byref(f), ctypes.byref(t)))
        return {"tma": bool(f.value & self.KERNELS_TMA), "fused_energy": bool(f.value & self.KERNELS_FUSED_ENERGY),
                "tma_passes": t.value}

    def autotune(self, params, repeats: int = 3, force: bool = False) -> str:
        """Time the plan candidates on these parameters (host array or CUDA
        tensor) and keep the fastest (cached per device and shape for the
        process); returns the candidates and the choice as text."""
        import torch

        p = params if isinstance(params, torch.Tensor) else torch.tensor(np.asarray(params, dtype=np.float64))
        p = p.to(device="cuda", dtype=torch.float64).reshape(-1).contiguous()
        check(self._lib.rsv_autotune(self._h, p.data_ptr(), p.numel(), int(repeats), 1 if force else 0,
                                     torch.cuda.current_stream().cuda_stream))
        text = self.describe()
        return text[text.index("autotune:"):] if "autotune:" in text else ""

    def describe(self) -> str:
        """The current plan (one line per kernel launch) and the last autotune report."""
        n = ctypes.c_size_t()
        check(self._lib.rsv_describe_backend(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        check(self._lib.rsv_describe_backend(self._h, buf, n.value + 1, ctypes.byref(n)))
        return buf.value.decode()

    def set_field(self, field: float) -> None:
        """Change the transverse field h (same circuit shape and buffers)."""
        check(self._lib.rsv_set_field(self._h, float(field)))
        self.field = float(field)

    def device_bytes(self) -> int:
        v = ctypes.c_size_t()
        check(self._lib.rsv_backend_info(self._h, None, None, None, ctypes.byref(v)))
        return int(v.value)


def describe_plan(num_qubits: int, num_layers: int, backward_mode: str = "auto") -> str:
    """Launch schedule of one energy_and_grad call (host only, no GPU needed)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(1 << 20)
    ln = ctypes.c_size_t()
    check(lib.rsv_describe_plan_mode(int(num_qubits), int(num_layers), Engine.BACKWARD_MODES[backward_mode],
                                     buf, len(buf), ctypes.byref(ln)))
    return buf.value.decode()

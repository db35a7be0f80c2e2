"""Mirror of the reference's Python backend wrapper for the standalone path.

Same names, argument meaning and error behaviour as zzEncounter/GPU_Simulation
``ring_ising/backends/standalone/config.py:19-117`` (``StandaloneBackendConfig``)
and ``ring_ising/backends/standalone/runtime.py:12-85``
(``RingIsingAdjointBackend``).  Like the reference, the wrapper drives the
compiled module ``standalone_backend._cuda_backend``; here that module is the
B200 drop-in built over librsv.so.
"""

from __future__ import annotations

import importlib
from dataclasses import dataclass

import numpy as np

# ring_ising/config.py:7-23
STANDALONE_GRADIENT_STRATEGIES = ("inverse_walk_cuQuantum", "structured_adjoint", "dense_scan")
STANDALONE_GRADIENT_STRATEGY_ALIASES = {"inverse_walk_cuquantum": "inverse_walk_cuQuantum"}
SUPPORTED_STANDALONE_GRADIENT_STRATEGIES = (
    *STANDALONE_GRADIENT_STRATEGIES,
    *STANDALONE_GRADIENT_STRATEGY_ALIASES,
)
STRUCTURED_ROTATION_CHUNK_WIDTH_MAX = 8
STRUCTURED_ADJOINT_GRADIENT_STRATEGIES = {"structured_adjoint"}
#: Device state buffers held per backend by this engine (psi, lambda, one scratch).
ENGINE_STATE_BUFFERS = 3


@dataclass(frozen=True)
class StandaloneBackendConfig:
    """Configuration for the standalone backend runtime (reference config.py:19-117)."""

    num_qubits: int
    layers: int
    field: float
    gradient_strategy: str
    structured_rotation_chunk_width: int = 8
    mode2_rotation_chunk_width: int | None = None
    double_buffer: bool = False

    @property
    def param_shape(self) -> tuple[int, int, int]:
        return (self.layers, self.num_qubits, 2)

    @property
    def num_params(self) -> int:
        return self.layers * self.num_qubits * 2

    @property
    def normalized_gradient_strategy(self) -> str:
        return STANDALONE_GRADIENT_STRATEGY_ALIASES.get(self.gradient_strategy, self.gradient_strategy)

    @property
    def effective_structured_rotation_chunk_width(self) -> int:
        if self.mode2_rotation_chunk_width is not None:
            return self.mode2_rotation_chunk_width
        return self.structured_rotation_chunk_width

    @property
    def statevector_nbytes(self) -> int:
        return (1 << self.num_qubits) * 16

    @property
    def dense_matrix_nbytes(self) -> int:
        dim = 1 << self.num_qubits
        return dim * dim * 16

    def estimated_gradient_state_buffers_for(self, strategy: str) -> int:
        """State buffers this engine allocates (the reference needs 4; this
        engine folds the CNOT ring into its passes and keeps 3)."""
        normalized = STANDALONE_GRADIENT_STRATEGY_ALIASES.get(strategy, strategy)
        if normalized not in STANDALONE_GRADIENT_STRATEGIES:
            raise ValueError("strategy must be one of STANDALONE_GRADIENT_STRATEGIES.")
        return ENGINE_STATE_BUFFERS

    def estimated_gradient_workspace_gib_for(self, strategy: str) -> float:
        padded = (1 << max(self.num_qubits, 12)) * 16
        return self.estimated_gradient_state_buffers_for(strategy) * padded / (1024**3)

    def validate(self) -> None:
        strategy = self.normalized_gradient_strategy
        if self.num_qubits < 2:
            raise ValueError("num_qubits must be at least 2.")
        if self.layers < 1:
            raise ValueError("layers must be at least 1.")
        if self.gradient_strategy not in SUPPORTED_STANDALONE_GRADIENT_STRATEGIES:
            raise ValueError(
                "gradient_strategy must be one of public strategies "
                f"{STANDALONE_GRADIENT_STRATEGIES!r}; accepted strategies are "
                f"{SUPPORTED_STANDALONE_GRADIENT_STRATEGIES!r}."
            )
        if strategy == "dense_scan" and self.num_qubits > 8:
            raise ValueError("dense_scan requires num_qubits <= 8.")
        chunk_width = self.effective_structured_rotation_chunk_width
        if chunk_width < 1:
            raise ValueError("structured_rotation_chunk_width must be at least 1.")
        if chunk_width > STRUCTURED_ROTATION_CHUNK_WIDTH_MAX:
            raise ValueError(
                f"structured_rotation_chunk_width must be at most {STRUCTURED_ROTATION_CHUNK_WIDTH_MAX}."
            )


class RingIsingAdjointBackend:
    """Python-facing entry point (reference runtime.py:12-85)."""

    def __init__(self, config: StandaloneBackendConfig) -> None:
        config.validate()
        self.config = config
        self.gradient_strategy = config.normalized_gradient_strategy
        self.uses_pennylane_gate_structure = self.gradient_strategy in {
            "inverse_walk_cuQuantum",
            "structured_adjoint",
        }
        self.estimated_workspace_gib = config.estimated_gradient_workspace_gib_for(self.gradient_strategy)
        self._backend = self._load_backend()
        self._cuda = self._backend.RingIsingCudaBackend(
            self.config.num_qubits,
            self.config.layers,
            float(self.config.field),
            self.gradient_strategy,
            int(self.config.effective_structured_rotation_chunk_width),
            bool(self.config.double_buffer),
        )

    @staticmethod
    def _load_backend():
        try:
            return importlib.import_module("standalone_backend._cuda_backend")
        except ImportError as exc:
            raise ImportError(
                "The B200 extension is not built yet. Run `python -m gpu_simulation_b200.build` first."
            ) from exc

    def _normalize_params(self, params: np.ndarray) -> np.ndarray:
        array = np.asarray(params, dtype=np.float64)
        if array.shape != self.config.param_shape:
            raise ValueError(f"Expected params with shape {self.config.param_shape}, got {array.shape}.")
        return np.ascontiguousarray(array.reshape(-1))

    def energy(self, params: np.ndarray) -> float:
        """Evaluate the Ising energy."""
        flat = self._normalize_params(params)
        raw = self._cuda.energy_and_grad(flat, False)
        return float(raw["energy"])

    def energy_and_grad(self, params: np.ndarray) -> tuple[float, np.ndarray]:
        """Evaluate the Ising energy and gradient."""
        flat = self._normalize_params(params)
        raw = self._cuda.energy_and_grad(flat)
        return float(raw["energy"]), np.asarray(raw["gradient"], dtype=np.float64).reshape(
            self.config.param_shape
        )

    def profile_energy_and_grad(self, params: np.ndarray) -> dict[str, object]:
        """Evaluate energy/gradient and return a stage timing breakdown."""
        flat = self._normalize_params(params)
        raw = self._cuda.energy_and_grad(flat, True, True)
        timings = {str(k): float(v) for k, v in dict(raw.get("timings_ms", {})).items()}
        return {
            "energy": float(raw["energy"]),
            "gradient": np.asarray(raw["gradient"], dtype=np.float64).reshape(self.config.param_shape),
            "timings_ms": timings,
        }

"""CPU oracle for the ring-Ising structured_adjoint path (test infrastructure).

This package is the CHECKER, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it.  It wraps ``librsv_oracle.so`` (``rsv_oracle.cpp``, a C++/OpenMP
restatement of the reference algorithm; each function there cites the
reference file:line it follows) and adds an exact-diagonalisation ground
energy for small rings.

Parity pins: the oracle is checked against the reference's own known answers
(``tests/golden/csv_known_answers.json``, the ``final_energy`` column of the
reference's 20-step training runs) and against the reference's CUDA extension
rebuilt for sm_100a (``oracle/_ref``, fixtures in ``tests/golden/``).
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "librsv_oracle.so"
_lib = None


def build() -> Path:
    """Compile librsv_oracle.so with the committed Makefile (g++ + OpenMP)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(_LIB_PATH))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.orc_set_num_threads.argtypes = [ctypes.c_int]
    lib.orc_set_num_threads.restype = None
    lib.orc_get_num_threads.argtypes = []
    lib.orc_get_num_threads.restype = ctypes.c_int
    lib.orc_ring_perm_closed.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int]
    lib.orc_ring_perm_closed.restype = ctypes.c_ulonglong
    lib.orc_ring_perm_loop.argtypes = [ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int]
    lib.orc_ring_perm_loop.restype = ctypes.c_ulonglong
    lib.orc_forward_state.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, dp]
    lib.orc_forward_state.restype = ctypes.c_int
    lib.orc_apply_hamiltonian.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp, dp]
    lib.orc_apply_hamiltonian.restype = ctypes.c_int
    lib.orc_energy_and_grad.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, ctypes.c_int, dp, dp,
    ]
    lib.orc_energy_and_grad.restype = ctypes.c_int
    _lib = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_num_threads(k: int) -> int:
    """Set the OpenMP thread count (0 = all host threads); returns the count in use."""
    lib = _load()
    lib.orc_set_num_threads(int(k))
    return int(lib.orc_get_num_threads())


def ring_perm(index: int, n: int, inverse: bool = False, closed_form: bool = True) -> int:
    """Ring-CNOT basis map P (or P^-1) of one index, closed form or bit loop."""
    lib = _load()
    fn = lib.orc_ring_perm_closed if closed_form else lib.orc_ring_perm_loop
    return int(fn(int(index), int(n), int(bool(inverse))))


def forward_state(n: int, layers: int, params, gate_level: bool = False) -> np.ndarray:
    """Final statevector (complex128, index bit w = wire w)."""
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
    if p.size != 2 * n * layers:
        raise ValueError("params size does not match n and layers")
    out = np.empty(2 << n, dtype=np.float64)
    if _load().orc_forward_state(n, layers, _dptr(p), int(gate_level), _dptr(out)) != 0:
        raise ValueError("oracle rejected the shape")
    return out.view(np.complex128)


def apply_hamiltonian(n: int, field: float, state: np.ndarray) -> tuple[np.ndarray, float]:
    """(H psi, <psi|H|psi>) for H = -sum Z_i Z_{i+1} - h sum X_i on a ring."""
    s = np.ascontiguousarray(np.asarray(state, dtype=np.complex128))
    if s.size != (1 << n):
        raise ValueError("state size does not match n")
    out = np.empty_like(s)
    e = np.zeros(1, dtype=np.float64)
    sv = s.view(np.float64)
    if _load().orc_apply_hamiltonian(n, float(field), _dptr(sv), _dptr(out.view(np.float64)), _dptr(e)) != 0:
        raise ValueError("oracle rejected the shape")
    return out, float(e[0])


def energy_and_grad(n: int, layers: int, field: float, params, mode: str = "structured_adjoint",
                    compute_gradient: bool = True):
    """Energy and gradient (flat f64[2 n L]) as the reference computes them.

    mode "structured_adjoint" follows the reference's structured schedule;
    "inverse_walk" is the gate-level adjoint (PennyLane gate order).
    """
    p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
    if p.size != 2 * n * layers:
        raise ValueError("params size does not match n and layers")
    m = {"structured_adjoint": 0, "inverse_walk": 1}[mode]
    e = np.zeros(1, dtype=np.float64)
    g = np.zeros(p.size, dtype=np.float64) if compute_gradient else None
    rc = _load().orc_energy_and_grad(
        n, layers, float(field), _dptr(p), m, _dptr(e), _dptr(g) if g is not None else None
    )
    if rc != 0:
        raise ValueError("oracle rejected the shape")
    return float(e[0]), g


def hamiltonian_sparse(n: int, field: float):
    """The ring-Ising Hamiltonian as a scipy CSR matrix (reference dense builder:
    cpp/ising_cuda_dense_helpers.inc:5-23)."""
    import scipy.sparse as sp

    S = 1 << n
    idx = np.arange(S, dtype=np.int64)
    mask = S - 1
    rot = ((idx << 1) & mask) | (idx >> (n - 1))
    walls = np.zeros(S, dtype=np.int64)
    x = (idx ^ rot) & mask
    for w in range(n):
        walls += (x >> w) & 1
    diag = 2.0 * walls - n
    rows = [idx]
    cols = [idx]
    vals = [diag]
    for w in range(n):
        rows.append(idx)
        cols.append(idx ^ (1 << w))
        vals.append(np.full(S, -float(field)))
    return sp.csr_matrix(
        (np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(S, S)
    )


def ground_energy_ed(n: int, field: float) -> float:
    """Exact ground energy by sparse Lanczos (n <= 16)."""
    import scipy.sparse.linalg as sla

    if n > 16:
        raise ValueError("exact diagonalisation is limited to n <= 16")
    H = hamiltonian_sparse(n, field)
    if n <= 10:
        return float(np.linalg.eigvalsh(H.toarray()).min())
    vals = sla.eigsh(H, k=1, which="SA", tol=1e-12)[0]
    return float(vals.min())


def ground_energy_free_fermion(n: int, field: float) -> float:
    """Periodic transverse-field Ising ground energy from the Pfeuty (1970)
    free-fermion solution, even-parity sector (antiperiodic fermion momenta
    k = (2m+1) pi / n):  E0 = -sum_k sqrt(1 + h^2 + 2 h cos k)  (J = 1)."""
    k = (2 * np.arange(n) + 1) * np.pi / n
    return float(-np.sum(np.sqrt(1.0 + field * field + 2.0 * field * np.cos(k))))


def initial_params(n: int, layers: int, seed: int = 7, init_scale: float = 0.3) -> np.ndarray:
    """Seeded init init_scale * N(0,1) of shape (L, n, 2), as the reference's
    ring_ising/params.py:8-20."""
    rng = np.random.default_rng(seed)
    return np.asarray(init_scale * rng.standard_normal((layers, n, 2)), dtype=np.float64)


def gradient_descent_final_energy(n: int, layers: int, field: float, steps: int,
                                  stepsize: float, seed: int = 7, init_scale: float = 0.3) -> float:
    """The reference's training loop (ring_ising/training/loop.py:75-139 with
    ring_ising/workflows/common.py:23-25): p <- p - stepsize * grad for `steps`
    steps, then energy(p) (workflows/standalone.py:133)."""
    p = initial_params(n, layers, seed, init_scale).reshape(-1)
    for _ in range(steps):
        _, g = energy_and_grad(n, layers, field, p)
        p = p - stepsize * g
    e, _ = energy_and_grad(n, layers, field, p, compute_gradient=False)
    return e


__all__ = [
    "apply_hamiltonian",
    "build",
    "energy_and_grad",
    "forward_state",
    "gradient_descent_final_energy",
    "ground_energy_ed",
    "ground_energy_free_fermion",
    "hamiltonian_sparse",
    "initial_params",
    "ring_perm",
    "set_num_threads",
]

if os.environ.get("RSV_ORACLE_THREADS"):
    set_num_threads(int(os.environ["RSV_ORACLE_THREADS"]))

"""ctypes binding of the engine's C ABI (include/rsv.h, include/rsv_shard.h, librsv.so).

The library is built in-tree (``python -m gpu_simulation_b200.build``).  There
is no CPU fallback: if librsv.so is missing or cannot be loaded, every entry
point raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "librsv.so"

RSV_OK = 0
RSV_ERR_INVALID_ARGUMENT = 1
RSV_ERR_STALE_STATE = 6

# Every function declared in include/rsv.h and include/rsv_shard.h, with its ctypes signature.
_c_double_p = ctypes.POINTER(ctypes.c_double)
_SIGNATURES = {
    "rsv_version": ([], ctypes.c_char_p),
    "rsv_last_error": ([], ctypes.c_char_p),
    "rsv_num_stages": ([], ctypes.c_int),
    "rsv_stage_name": ([ctypes.c_int], ctypes.c_char_p),
    "rsv_create": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_int,
                    ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rsv_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rsv_energy_and_grad": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_energy_and_grad_device": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_forward_device": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                            ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_void_p], ctypes.c_int),
    "rsv_backward_device": ([ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p],
                             ctypes.c_int),
    "rsv_profile_energy_and_grad": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_benchmark_forward_graph": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                                     _c_double_p, _c_double_p], ctypes.c_int),
    "rsv_energy_and_grad_noalloc": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                                    ctypes.c_int),
    "rsv_set_launch_timing": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rsv_kernel_launches": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_launch_stats": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                         ctypes.c_int),
    "rsv_set_field": ([ctypes.c_void_p, ctypes.c_double], ctypes.c_int),
    "rsv_zgemm_batched": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                           ctypes.c_void_p], ctypes.c_int),
    "rsv_set_backward_mode": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rsv_set_analytic_layers": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rsv_set_kernels": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rsv_batch_set_cluster": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rsv_batch_cluster": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "rsv_autotune": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                      ctypes.c_void_p], ctypes.c_int),
    "rsv_describe_backend": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)],
                             ctypes.c_int),
    "rsv_kernels": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "rsv_analytic_layers": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
                            ctypes.c_int),
    "rsv_backward_mode": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "rsv_describe_plan_mode": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
                                ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "rsv_backend_info": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                          ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "rsv_describe_plan": ([ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
                           ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "rsv_ring_map": ([ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int], ctypes.c_ulonglong),
    "rsv_batch_create": ([ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rsv_batch_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "rsv_batch_set_circuits": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p], ctypes.c_int),
    "rsv_batch_info": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_size_t),
                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_size_t)], ctypes.c_int),
    "rsv_batch_set_active_slots": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rsv_batch_run_device": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_void_p], ctypes.c_int),
    "rsv_batch_energy_and_grad": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_mlp_num_weights": ([ctypes.c_int, ctypes.c_void_p], ctypes.c_size_t),
    "rsv_mlp_work_floats": ([ctypes.c_int, ctypes.c_void_p, ctypes.c_int], ctypes.c_size_t),
    "rsv_mlp_scratch_floats": ([ctypes.c_int, ctypes.c_void_p, ctypes.c_int], ctypes.c_size_t),
    "rsv_mlp_forward": ([ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_mlp_backward": ([ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.c_void_p], ctypes.c_int),
    "rsv_mlp_mse": ([ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                     ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_adam_f32": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                      ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                      ctypes.c_void_p], ctypes.c_int),
    "rsv_adam_f64": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                      ctypes.c_void_p], ctypes.c_int),
    "rsv_gd_step_f64": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p,
                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_adam_vqe_step_f64": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    # include/rsv_shard.h
    "rsv_shard_check": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "rsv_shard_scratch_doubles": ([ctypes.c_int, ctypes.c_int], ctypes.c_size_t),
    "rsv_shard_coef": ([ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                       ctypes.c_int),
    "rsv_shard_init": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
                       ctypes.c_int),
    "rsv_shard_rotate_local": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p], ctypes.c_int),
    "rsv_shard_rotate_local_adjoint": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p], ctypes.c_int),
    "rsv_shard_energy_local": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_shard_ring_pack": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_shard_ring_unpack": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p], ctypes.c_int),
    "rsv_shard_ring_pack_adjoint": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rsv_shard_ring_unpack_adjoint": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
}

_lib = None


class EngineError(RuntimeError):
    """A CUDA or internal failure reported by the engine."""


def load_library() -> ctypes.CDLL:
    """Load librsv.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built; run `python -m gpu_simulation_b200.build` "
            "(the engine has no CPU fallback)."
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(status: int) -> None:
    """Raise ValueError / EngineError for a non-zero rsv_status."""
    if status == RSV_OK:
        return
    msg = load_library().rsv_last_error().decode()
    if status == RSV_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise EngineError(f"rsv status {status}: {msg}")

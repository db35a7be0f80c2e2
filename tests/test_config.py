"""StandaloneBackendConfig validation, mirroring the reference's config tests
(tests/test_backends_parity.py:237-292 of zzEncounter/GPU_Simulation)."""

from __future__ import annotations

import pytest

from gpu_simulation_b200.backend import StandaloneBackendConfig

REMOVED_MODES = ("inverse_walk", "ryrz_fused", "mode2", "save_param_states", "checkpoint")


@pytest.mark.parametrize("mode", REMOVED_MODES)
def test_removed_modes_are_rejected(mode):
    with pytest.raises(ValueError):
        StandaloneBackendConfig(4, 2, 1.0, mode).validate()


def test_dense_scan_qubit_limit():
    StandaloneBackendConfig(8, 2, 1.0, "dense_scan").validate()
    with pytest.raises(ValueError):
        StandaloneBackendConfig(9, 2, 1.0, "dense_scan").validate()


@pytest.mark.parametrize("width,ok", [(0, False), (1, True), (8, True), (9, False)])
def test_chunk_width_range(width, ok):
    cfg = StandaloneBackendConfig(10, 2, 1.0, "structured_adjoint", structured_rotation_chunk_width=width)
    if ok:
        cfg.validate()
    else:
        with pytest.raises(ValueError):
            cfg.validate()


def test_alias_and_shapes():
    cfg = StandaloneBackendConfig(6, 3, 0.5, "inverse_walk_cuquantum", mode2_rotation_chunk_width=4)
    cfg.validate()
    assert cfg.normalized_gradient_strategy == "inverse_walk_cuQuantum"
    assert cfg.effective_structured_rotation_chunk_width == 4
    assert cfg.param_shape == (3, 6, 2)
    assert cfg.num_params == 36
    assert cfg.statevector_nbytes == 64 * 16


def test_workspace_estimate_counts_three_padded_buffers():
    cfg = StandaloneBackendConfig(30, 4, 1.0, "structured_adjoint")
    assert cfg.estimated_gradient_state_buffers_for("structured_adjoint") == 3
    assert abs(cfg.estimated_gradient_workspace_gib_for("structured_adjoint") - 48.0) < 1e-9
    small = StandaloneBackendConfig(4, 1, 1.0, "structured_adjoint")
    assert small.estimated_gradient_workspace_gib_for("structured_adjoint") == 3 * 4096 * 16 / 1024**3

"""The allocation-free entry point (rsv_energy_and_grad_noalloc).

It serves callers that must not allocate device memory themselves (their
memory belongs to another allocator, or an allocation and its implicit device
synchronisation are not allowed where they run): all scratch lives in one
fixed workspace inside the library.  These tests call it through the C ABI
and compare it with the regular device entry point, on consecutive calls --
including a small circuit after a larger one, because the shared workspace
keeps the previous call's contents.  This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from gpu_simulation_b200 import Engine, _lib

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _noalloc(n, L, h, params):
    import torch

    lib = _lib.load_library()
    dp = torch.tensor(params, device="cuda")
    de = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    dg = torch.full_like(dp, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.rsv_energy_and_grad_noalloc(n, L, h, dp.data_ptr(), dp.numel(), de.data_ptr(), dg.data_ptr(),
                                         stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    return de.item(), dg.cpu().numpy()


def _regular(n, L, h, params):
    import torch

    eng = Engine(n, L, h)
    dp = torch.tensor(params, device="cuda")
    de = torch.empty(1, dtype=torch.float64, device="cuda")
    dg = torch.empty_like(dp)
    eng.energy_and_grad_device(dp, de, dg)
    torch.cuda.synchronize()
    out = (de.item(), dg.cpu().numpy())
    eng.close()
    return out


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    cases = [(14, 2, 0.9, 1), (6, 3, 1.1, 2), (12, 4, 1.0, 3)]
    for n, L, h, seed in cases:
        p = np.random.default_rng(seed).uniform(0, 2 * np.pi, 2 * n * L)
        e0, g0 = _noalloc(n, L, h, p)
        e1, g1 = _regular(n, L, h, p)
        assert abs(e0 - e1) < TOL, (n, L, e0, e1)
        np.testing.assert_allclose(g0, g1, atol=TOL, rtol=0)


def test_noalloc_at_its_stated_limit_and_energy_only():
    # n=16, L=64 is the largest circuit the fixed workspace takes (the largest
    # carve of state buffers, tables and per-CTA records); then the same call
    # for the energy alone (no gradient pointer), and a small circuit after it
    import torch

    lib = _lib.load_library()
    for n, L, h, seed in ((16, 64, 0.8, 11), (16, 63, 1.3, 12), (13, 64, 1.0, 13), (3, 64, 0.6, 14)):
        p = np.random.default_rng(seed).uniform(0, 2 * np.pi, 2 * n * L)
        e0, g0 = _noalloc(n, L, h, p)
        e1, g1 = _regular(n, L, h, p)
        assert abs(e0 - e1) < TOL, (n, L, e0, e1)
        np.testing.assert_allclose(g0, g1, atol=TOL, rtol=0)
        dp = torch.tensor(p, device="cuda")
        de = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(lib.rsv_energy_and_grad_noalloc(n, L, h, dp.data_ptr(), dp.numel(), de.data_ptr(), None,
                                                   torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert abs(de.item() - e1) < TOL, (n, L, de.item(), e1)


def test_noalloc_every_size_up_to_the_limit():
    # every qubit count up to the limit at a few depths, so every carve the
    # workspace can be asked for is exercised
    for n in range(2, 17):
        for L in (1, 2, 5, 17, 64):
            p = np.random.default_rng(100 * n + L).uniform(0, 2 * np.pi, 2 * n * L)
            e0, g0 = _noalloc(n, L, 1.0, p)
            e1, g1 = _regular(n, L, 1.0, p)
            assert abs(e0 - e1) < TOL, (n, L, e0, e1)
            np.testing.assert_allclose(g0, g1, atol=TOL, rtol=0)


def test_noalloc_rejects_sizes_beyond_its_workspace():
    import torch

    lib = _lib.load_library()
    n, L = 17, 2
    dp = torch.zeros(2 * n * L, dtype=torch.float64, device="cuda")
    de = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = lib.rsv_energy_and_grad_noalloc(n, L, 1.0, dp.data_ptr(), dp.numel(), de.data_ptr(), None, 0)
    assert rc == _lib.RSV_ERR_INVALID_ARGUMENT
    assert "num_qubits <= 16" in lib.rsv_last_error().decode()
    n, L = 8, 65
    dp = torch.zeros(2 * n * L, dtype=torch.float64, device="cuda")
    rc = lib.rsv_energy_and_grad_noalloc(n, L, 1.0, dp.data_ptr(), dp.numel(), de.data_ptr(), None, 0)
    assert rc == _lib.RSV_ERR_INVALID_ARGUMENT
    assert "num_layers <= 64" in lib.rsv_last_error().decode()


def test_noalloc_on_every_visible_device():
    # the workspace address and the kernels' shared-memory limits are set up
    # per device: a call on each visible GPU in turn must match the regular
    # entry point on that GPU (skipped with one GPU)
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    n, L, h = 14, 3, 0.8
    p = np.random.default_rng(77).uniform(0, 2 * np.pi, 2 * n * L)
    for dev in range(torch.cuda.device_count()):
        with torch.cuda.device(dev):
            e0, g0 = _noalloc(n, L, h, p)
            e1, g1 = _regular(n, L, h, p)
        assert abs(e0 - e1) < TOL, (dev, e0, e1)
        np.testing.assert_allclose(g0, g1, atol=TOL, rtol=0)

"""dense_scan (n <= 8): the batched complex GEMM on FP64 tensor cores against
numpy and against cuBLAS's speed, and the dense energy and gradient against
the oracle at 1e-10."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from gpu_simulation_b200 import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-10


def zgemm(a, b):
    import torch

    from gpu_simulation_b200._lib import check, load_library

    lib = load_library()
    ta = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tb = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    tc = torch.empty_like(ta)
    check(lib.rsv_zgemm_batched(ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), a.shape[-1], a.shape[0],
                                torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return tc.cpu().numpy()


@pytest.mark.parametrize("dim,batch", [(4, 3), (16, 2), (32, 3), (64, 2), (96, 1), (256, 3)])
def test_zgemm_matches_numpy(dim, batch):
    rng = np.random.default_rng(dim + batch)
    a = rng.standard_normal((batch, dim, dim)) + 1j * rng.standard_normal((batch, dim, dim))
    b = rng.standard_normal((batch, dim, dim)) + 1j * rng.standard_normal((batch, dim, dim))
    c = zgemm(a, b)
    assert np.max(np.abs(c - a @ b)) < 1e-12 * dim


@pytest.mark.parametrize("n,L,h", [(2, 1, 0.7), (2, 3, 1.0), (3, 2, 1.1), (4, 5, 0.4), (5, 1, 1.0), (5, 4, 1.2),
                                   (6, 3, 0.9), (7, 2, 1.5), (8, 1, 1.0), (8, 3, 1.0), (8, 6, 0.6)])
def test_dense_scan_matches_oracle(n, L, h):
    p = np.random.default_rng(70 + 11 * n + L).uniform(0.0, 2.0 * np.pi, 2 * n * L)
    e_ref, g_ref = oracle.energy_and_grad(n, L, h, p)
    eng = Engine(n, L, h, gradient_strategy="dense_scan")
    e, g = eng.energy_and_grad(p)
    assert abs(e - e_ref) < TOL, (e, e_ref)
    np.testing.assert_allclose(g, g_ref, atol=TOL, rtol=0)
    assert abs(eng.energy(p) - e) < 1e-13
    prof = eng.profile_energy_and_grad(p)
    assert abs(prof["energy"] - e) < 1e-13


def test_dense_scan_rejects_large_n():
    with pytest.raises(ValueError):
        Engine(9, 2, 1.0, gradient_strategy="dense_scan")


def test_zgemm_speed_against_cublas():
    # the reference builds its product tree with cublasZgemmStridedBatched;
    # torch's complex128 bmm calls the same library
    import torch

    from gpu_simulation_b200._lib import check, load_library

    lib = load_library()
    dim, batch = 256, 8
    a = torch.randn(batch, dim, dim, dtype=torch.complex128, device="cuda")
    b = torch.randn(batch, dim, dim, dtype=torch.complex128, device="cuda")
    c = torch.empty_like(a)
    s = torch.cuda.current_stream().cuda_stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for _ in range(3):
        torch.bmm(a, b, out=c)
        check(lib.rsv_zgemm_batched(a.data_ptr(), b.data_ptr(), c.data_ptr(), dim, batch, s))
    ev[0].record()
    for _ in range(20):
        torch.bmm(a, b, out=c)
    ev[1].record()
    for _ in range(20):
        check(lib.rsv_zgemm_batched(a.data_ptr(), b.data_ptr(), c.data_ptr(), dim, batch, s))
    ev[2].record()
    ev[2].synchronize()
    cublas_ms = ev[0].elapsed_time(ev[1]) / 20
    ours_ms = ev[1].elapsed_time(ev[2]) / 20
    flops = 8.0 * batch * dim ** 3
    print(f"zgemm {batch}x{dim}^3: cuBLAS {cublas_ms:.4f} ms ({flops / cublas_ms / 1e9:.2f} TF/s), "
          f"ours {ours_ms:.4f} ms ({flops / ours_ms / 1e9:.2f} TF/s)")
    assert torch.allclose(c, torch.bmm(a, b), atol=1e-9, rtol=0)

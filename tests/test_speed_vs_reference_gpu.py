"""Speed check against the reference's own structured_adjoint extension
rebuilt for sm_100a (oracle/_ref), on the same GPU and inputs: the engine
must be faster, and both must agree at 1e-10.  Timings are printed and, when
RSV_SPEED_LOG is set, appended to that file as JSON lines."""

from __future__ import annotations

import json
import os
import time

import numpy as np
import pytest

from gpu_simulation_b200 import Engine
from tests.refmod import load_reference_module

pytestmark = pytest.mark.gpu

ref = load_reference_module()


def _time(fn, reps):
    fn()
    t0 = time.perf_counter()
    for _ in range(reps):
        r = fn()
    return (time.perf_counter() - t0) / reps * 1e3, r


@pytest.mark.skipif(ref is None, reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("n,L,reps", [(20, 4, 10), (24, 4, 5), (26, 4, 2)])
def test_engine_is_faster_than_reference(n, L, reps):
    p = np.random.default_rng(7).uniform(0, 2 * np.pi, 2 * n * L)
    rb = ref.RingIsingCudaBackend(n, L, 1.0, "structured_adjoint", 8, False)
    ms_ref, r = _time(lambda: rb.energy_and_grad(p, True, False), reps)
    del rb
    eng = Engine(n, L, 1.0)
    ms_new, (e, g) = _time(lambda: eng.energy_and_grad(p), reps)
    eng.close()
    assert abs(e - r["energy"]) < 1e-10
    np.testing.assert_allclose(g, np.asarray(r["gradient"]), atol=1e-10, rtol=0)
    rec = {"n": n, "L": L, "reference_ms": ms_ref, "engine_ms": ms_new, "speedup": ms_ref / ms_new}
    print(json.dumps(rec))
    if os.environ.get("RSV_SPEED_LOG"):
        with open(os.environ["RSV_SPEED_LOG"], "a") as fh:
            fh.write(json.dumps(rec) + "\n")
    assert ms_new < ms_ref


@pytest.mark.skipif(ref is None, reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("strategy,n,L,reps", [("dense_scan", 8, 8, 10), ("dense_scan", 6, 16, 10),
                                               ("inverse_walk_cuQuantum", 16, 4, 3)])
def test_other_strategies_against_reference(strategy, n, L, reps):
    # dense_scan on both sides: the reference's cuBLAS product tree vs the
    # FP64-MMA tree.  The reference's gate-level path needs cuStateVec, which
    # the rebuild replaces by a stand-in, so the gate-level walk is checked
    # (and timed) against the reference's structured path instead.
    p = np.random.default_rng(3).uniform(0, 2 * np.pi, 2 * n * L)
    ref_strategy = strategy if strategy == "dense_scan" else "structured_adjoint"
    rb = ref.RingIsingCudaBackend(n, L, 1.0, ref_strategy, 8, False)
    ms_ref, r = _time(lambda: rb.energy_and_grad(p, True, False), reps)
    del rb
    eng = Engine(n, L, 1.0, gradient_strategy=strategy)
    ms_new, (e, g) = _time(lambda: eng.energy_and_grad(p), reps)
    eng.close()
    assert abs(e - r["energy"]) < 1e-10
    np.testing.assert_allclose(g, np.asarray(r["gradient"]), atol=1e-10, rtol=0)
    rec = {"strategy": strategy, "n": n, "L": L, "reference_ms": ms_ref, "engine_ms": ms_new,
           "speedup": ms_ref / ms_new}
    print(json.dumps(rec))
    if os.environ.get("RSV_SPEED_LOG"):
        with open(os.environ["RSV_SPEED_LOG"], "a") as fh:
            fh.write(json.dumps(rec) + "\n")

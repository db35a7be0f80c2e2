"""Pins of the CPU oracle (no GPU): the reference's own known answers, two
independent statements of the ring permutation, gate-level vs structured
adjoint, central finite differences and exact diagonalisation."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).parent / "golden"


def test_known_answers_from_reference_training_runs():
    """20 GD steps (stepsize 0.08, seed 7, init 0.3 N(0,1), h=1, L=2) reproduce
    the reference's published final energies (both of its GPU strategies)."""
    data = json.loads((GOLDEN / "csv_known_answers.json").read_text())
    proto = data["protocol"]
    for n in (8, 9, 10, 11, 12, 13, 14):
        ref = data["final_energy"][str(n)]
        e = oracle.gradient_descent_final_energy(
            n, proto["layers"], proto["field"], proto["steps"], proto["stepsize"],
            proto["seed"], proto["init_scale"],
        )
        for method, value in ref.items():
            assert abs(e - value) < 1e-9, (n, method, e, value)


def test_ring_permutation_closed_form_matches_gate_loop():
    for n in range(2, 11):
        for i in range(1 << n):
            p = oracle.ring_perm(i, n)
            assert p == oracle.ring_perm(i, n, closed_form=False)
            assert oracle.ring_perm(p, n, inverse=True) == i
            assert oracle.ring_perm(p, n, inverse=True, closed_form=False) == i


def test_structured_matches_gate_level_inverse_walk():
    rng = np.random.default_rng(11)
    for n, L, h in [(2, 1, 0.7), (3, 3, 1.0), (5, 2, 1.1), (8, 3, 0.4), (10, 2, 1.7)]:
        p = rng.uniform(0, 2 * np.pi, 2 * n * L)
        e1, g1 = oracle.energy_and_grad(n, L, h, p)
        e2, g2 = oracle.energy_and_grad(n, L, h, p, mode="inverse_walk")
        assert abs(e1 - e2) < 1e-12
        np.testing.assert_allclose(g1, g2, atol=1e-12, rtol=0)


def test_state_matches_gate_level_state():
    rng = np.random.default_rng(5)
    for n, L in [(4, 2), (7, 3)]:
        p = rng.uniform(0, 2 * np.pi, 2 * n * L)
        np.testing.assert_allclose(
            oracle.forward_state(n, L, p), oracle.forward_state(n, L, p, gate_level=True), atol=1e-13
        )


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(2)
    n, L, h = 6, 3, 0.9
    p = rng.uniform(0, 2 * np.pi, 2 * n * L)
    _, g = oracle.energy_and_grad(n, L, h, p)
    step = 1e-5
    for k in rng.choice(p.size, 8, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[k] += step
        pm[k] -= step
        fd = (oracle.energy_and_grad(n, L, h, pp, compute_gradient=False)[0]
              - oracle.energy_and_grad(n, L, h, pm, compute_gradient=False)[0]) / (2 * step)
        assert abs(fd - g[k]) < 1e-7


@pytest.mark.parametrize("n,h", [(4, 0.5), (8, 1.0), (12, 1.3), (14, 0.7)])
def test_exact_diagonalisation_matches_free_fermions(n, h):
    assert abs(oracle.ground_energy_ed(n, h) - oracle.ground_energy_free_fermion(n, h)) < 1e-9


def test_variational_energy_bounded_by_ground_energy():
    rng = np.random.default_rng(4)
    n, L, h = 8, 3, 1.0
    e0 = oracle.ground_energy_ed(n, h)
    for _ in range(5):
        e, _ = oracle.energy_and_grad(n, L, h, rng.uniform(0, 2 * np.pi, 2 * n * L), compute_gradient=False)
        assert e >= e0 - 1e-12


def test_hamiltonian_matches_sparse_matrix():
    rng = np.random.default_rng(8)
    n, h = 7, 1.2
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    lam, e = oracle.apply_hamiltonian(n, h, psi)
    H = oracle.hamiltonian_sparse(n, h)
    np.testing.assert_allclose(lam, H @ psi, atol=1e-12)
    assert abs(e - np.vdot(psi, H @ psi).real) < 1e-9


def test_oracle_matches_reference_golden_vectors():
    """Golden vectors produced by the reference's own CUDA extension (rebuilt
    for sm_100a, tests/golden/make_ref_golden.py) pin the oracle at 1e-10."""
    data = json.loads((GOLDEN / "ref_golden.json").read_text())
    assert len(data["cases"]) >= 15
    for case in data["cases"]:
        n, L, h = case["n"], case["L"], case["h"]
        if n > 18:
            continue  # the larger cases are checked on the GPU
        p = np.random.default_rng(case["seed"]).uniform(0.0, 2.0 * np.pi, 2 * n * L)
        e, g = oracle.energy_and_grad(n, L, h, p)
        assert abs(e - case["energy"]) < 1e-10, (n, L, e, case["energy"])
        np.testing.assert_allclose(g, np.asarray(case["gradient"]), atol=1e-10, rtol=0)

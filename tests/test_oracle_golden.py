"""The oracle is pinned to the reference's own known-answer values.

Golden values: ForceConstants.jl test/runtests.jl:109-136 ("LJ Values"),
extracted to tests/golden/lj_values.json by tests/golden/make_golden.py.
"""
import json
import os

import numpy as np
import pytest

from conftest import AR, fcc_system

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "lj_values.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ar256(oracle):
    s = fcc_system((4, 4, 4))
    tol = 1e-8
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], tol)
    psi = oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], tol)
    return s, ifc2, psi


def _close(actual, expected, rtol):
    # Julia's ≈ on scalars: |x - y| <= rtol * max(|x|, |y|), exact for 0.
    if expected == 0.0:
        return actual == 0.0
    return abs(actual - expected) <= rtol * max(abs(actual), abs(expected))


def test_ifc2_golden(ar256, golden):
    _, ifc2, _ = ar256
    for g in golden["ifc2"]:
        i, j = (x - 1 for x in g["index_1based"])
        assert _close(ifc2[i, j], g["value"], golden["rtol"]), (g, ifc2[i, j])


def test_ifc3_golden(ar256, golden):
    _, _, psi = ar256
    assert len(golden["ifc3"]) == 7
    for g in golden["ifc3"]:
        i, j, k = (x - 1 for x in g["index_1based"])
        assert _close(psi[i, j, k], g["value"], golden["rtol"]), (g, psi[i, j, k])


def test_ifc2_asr_and_symmetry(ar256):
    # runtests.jl:123-124: asr_satisfied and issymmetric
    s, ifc2, _ = ar256
    from fcb200.ifc import asr_satisfied
    assert asr_satisfied(ifc2, s.n_atoms, 3, 1e-8)
    assert np.array_equal(ifc2, ifc2.T)


def test_ifc3_permutation_symmetry_and_asr(ar256):
    _, _, psi = ar256
    # Ψ is symmetric under index permutations up to rounding of the scatter.
    for perm in [(1, 0, 2), (2, 1, 0), (0, 2, 1)]:
        assert np.max(np.abs(psi - psi.transpose(perm))) < 1e-12
    # Acoustic sum rule on the last index: Σ_k Ψ[i,j,k] = 0 for the FCC lattice.
    s = psi.reshape(768, 768, 256, 3).sum(axis=2)
    assert np.max(np.abs(s)) < 1e-10


def test_oracle_cutoff_assert(oracle):
    s = fcc_system((1, 1, 1))
    with pytest.raises(ValueError):
        oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)


def test_oracle_mcc3_blocked_equals_full(oracle):
    rng = np.random.default_rng(3)
    n = 12
    psi = rng.normal(size=(n, n, n))
    phi = np.linalg.qr(rng.normal(size=(n, n)))[0]
    full = oracle.mcc3(psi, phi)
    ref = np.einsum("ijk,in,jm,kl->nml", psi, phi, phi, phi)
    assert np.allclose(full, ref, atol=1e-12)
    for b in (3, 4, 6, 12):
        assert np.allclose(oracle.mcc3_blocked(psi, phi, b), full, atol=1e-12)
    with pytest.raises(ValueError):
        oracle.mcc3_blocked(psi, phi, 5)


def test_oracle_mass_weight(oracle):
    s = fcc_system((2, 2, 2), std=0.05, seed=1)
    psi = oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    m = np.linspace(30.0, 50.0, s.n_atoms)
    w = oracle.mass_weight_third_order(psi.copy(order="F"), m)
    mm = np.repeat(m, 3)
    expect = psi / np.sqrt(mm[:, None, None] * mm[None, :, None] * mm[None, None, :])
    assert np.allclose(w, expect, rtol=1e-15, atol=0)

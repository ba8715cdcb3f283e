"""Adjoint of the LJ snapshot on the GPU (fcb200_mcc3_adjoint_lj).

Checks ∂L/∂positions, ∂L/∂σ, ∂L/∂ε for L = Σ W·K3 (φ frozen) against
(1) the FP64 pair-form adjoint of the oracle and (2) central finite
differences of the FP64 reference path (h = 1e-5 Å for positions, 1e-6
relative for σ and ε).  Tolerance: 1e-6 relative (normwise over the checked
components) for the FP32 and TF32×3 forms of G; 1e-4 for BF16×3.
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu
TOL = {"fp32": 1e-6, "tf32x3": 1e-6, "bf16x3": 1e-4}


@pytest.fixture(scope="module")
def small(fcb, oracle):
    s = fcc_system((2, 2, 2), 0.05, 3)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    phi32 = np.asfortranarray(phi.astype(np.float32))
    M = 24
    W = np.asfortranarray(np.random.default_rng(5).normal(size=(M, M, M)).astype(np.float32))
    ref = oracle.lj_adjoint(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, s.masses,
                            phi32.astype(np.float64), W.astype(np.float64))
    return s, pot, calc, phi32, W, ref


@pytest.mark.parametrize("precision", ["fp32", "tf32x3", "bf16x3"])
def test_adjoint_vs_fp64_pair_form(fcb, cuda_device, small, precision):
    from fcb200.adjoint import mcc3_adjoint_lj
    s, pot, calc, phi32, W, (gpos, gs, ge, L) = small
    out = mcc3_adjoint_lj(s, pot, calc, phi32, W, precision=precision)
    tol = TOL[precision]
    assert np.max(np.abs(out["dpos"] - gpos)) <= tol * np.max(np.abs(gpos))
    assert abs(out["dsigma"] - gs) <= tol * abs(gs)
    assert abs(out["deps"] - ge) <= tol * abs(ge)
    assert abs(out["L"] - L) <= tol * abs(L)


def test_adjoint_vs_central_differences(fcb, oracle, cuda_device, small):
    from fcb200.adjoint import mcc3_adjoint_lj
    s, pot, calc, phi32, W, _ = small
    out = mcc3_adjoint_lj(s, pot, calc, phi32, W, precision="tf32x3")
    phi64, W64 = phi32.astype(np.float64), W.astype(np.float64)

    def L(pos, sg=pot.sigma, ep=pot.eps):
        return oracle.mcc3_loss_lj(pos, s.box_sizes, sg, ep, pot.r_cut, s.masses, phi64, W64)

    h = 1e-5
    comps = [(0, 0), (3, 1), (7, 2), (15, 0), (31, 1), (20, 2)]
    fd, ad = [], []
    for a, d in comps:
        p = s.positions.copy()
        p[a, d] += h
        lp = L(p)
        p[a, d] -= 2 * h
        fd.append((lp - L(p)) / (2 * h))
        ad.append(out["dpos"][a, d])
    fd, ad = np.array(fd), np.array(ad)
    assert np.max(np.abs(fd - ad)) <= 1e-6 * np.max(np.abs(fd))
    hs = pot.sigma * 1e-6
    fds = (L(s.positions, pot.sigma + hs) - L(s.positions, pot.sigma - hs)) / (2 * hs)
    assert abs(fds - out["dsigma"]) <= 1e-6 * abs(fds)
    he = pot.eps * 1e-6
    fde = (L(s.positions, pot.sigma, pot.eps + he) - L(s.positions, pot.sigma, pot.eps - he)) / (2 * he)
    assert abs(fde - out["deps"]) <= 1e-6 * abs(fde)

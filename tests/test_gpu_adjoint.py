"""Adjoint of the LJ snapshot on the GPU (fcb200_mcc3_adjoint_lj).

Checks ∂L/∂positions, ∂L/∂σ, ∂L/∂ε for L = Σ W·K3 (φ frozen) against
(1) the FP64 pair-form adjoint of the oracle and (2) central finite
differences of the FP64 reference path (h = 1e-5 Å for positions, 1e-6
relative for σ and ε), on a 32-atom cell and at the differentiation
configuration (256 atoms, W over the first 256 modes, all 768 position
components).  Tolerance against the oracle's pair form on the small cell:
1e-8 relative (normwise over the checked components) for the FP64 form of G
(its mode products on the FP64 tensor cores, with partial 128-row and
128-mode tiles at n = 96 and M = 24), 1e-6 for the FP32 and TF32×3 forms,
1e-4 for BF16×3.  At the differentiation configuration: 1e-6 of
central differences for the FP64 form of G (the default); the FP32 and TF32×3
forms, limited by their own rounding of G, within 5e-6 and 1e-5 of it.
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-8, "fp32": 1e-6, "tf32x3": 1e-6, "bf16x3": 1e-4}


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


@pytest.mark.parametrize("precision", ["fp64", "fp32", "tf32x3", "bf16x3"])
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


def _config5_reference(fcb, cuda_device):
    """The differentiation configuration: the 256-atom displaced cell of the
    precision configuration (std 0.05 Å, seed 1234, tol 1e-12), φ frozen (FP32
    modes of its dynamical matrix, from the device), W ~ N(0,1) over the first
    256 modes on every axis (seeded).  L is linear in the mass-weighted Ψ,
    L(x) = Σ G[i,j,k] Ψ(x)[i,j,k] / sqrt(m_i m_j m_k) with G = W ×₁φᵀ ×₂φᵀ ×₃φᵀ,
    so the reference L is evaluated with G formed once in FP64 (torch, on the
    device) and the GPU's FP64 Ψ, which is bit-exact to the oracle."""
    import torch
    s = fcc_system((4, 4, 4), 0.05, 1234)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    M = 256
    dyn = fcb.dynamical_matrix(s, pot, calc, device="cuda")
    _, _, phi = fcb.get_modes(dyn, 3, phi32=True)
    W32 = np.asfortranarray(np.random.default_rng(2025).normal(size=(M, M, M)).astype(np.float32))
    ph = phi[:, :M].double()
    W = torch.from_numpy(np.ascontiguousarray(W32.astype(np.float64))).to(cuda_device)   # [p,q,s] logical
    g = torch.tensordot(ph, W, dims=([1], [0]))          # [i, q, s]
    g = torch.tensordot(g, ph, dims=([1], [1]))          # [i, s, j]
    g = torch.tensordot(g, ph, dims=([1], [1]))          # [i, j, k]
    w = torch.from_numpy(np.repeat(s.masses, 3) ** -0.5).to(cuda_device)
    gw = g * w[:, None, None] * w[None, :, None] * w[None, None, :]
    del g
    flat = gw.permute(2, 1, 0).contiguous().reshape(-1)  # column-major memory order, as Ψ
    del gw

    def L(pos, sigma=pot.sigma, eps=pot.eps):
        sys_ = fcb.SuperCellSystem(pos, s.masses, s.box_sizes)
        psi = fcb.third_order(sys_, fcb.LJ(sigma, eps, pot.r_cut), calc, device="cuda").values
        return float(torch.dot(psi.permute(2, 1, 0).reshape(-1), flat))

    return s, pot, calc, phi.cpu().numpy(), W32, L


def test_adjoint_config5_vs_central_differences(fcb, cuda_device):
    """All 768 position components, σ and ε of the differentiation
    configuration against central differences (h = 1e-5 Å; 1e-6 relative for
    σ and ε) of the FP64 L, with G formed in FP64 by the adjoint.  Tolerance
    1e-6 relative: max over the components of |AD − FD| / max |FD|, and
    |AD − FD| / |FD| for σ and ε."""
    from fcb200.adjoint import mcc3_adjoint_lj
    s, pot, calc, phi32, W32, L = _config5_reference(fcb, cuda_device)
    out = mcc3_adjoint_lj(s, pot, calc, phi32, W32, precision="fp64")
    L0 = L(s.positions)
    assert abs(out["L"] - L0) <= 1e-10 * abs(L0)
    h = 1e-5
    fd = np.zeros_like(s.positions)
    for a in range(s.n_atoms):
        for d in range(3):
            p = s.positions.copy()
            p[a, d] += h
            lp = L(p)
            p[a, d] -= 2 * h
            fd[a, d] = (lp - L(p)) / (2 * h)
    err = np.max(np.abs(out["dpos"] - fd)) / np.max(np.abs(fd))
    assert err <= 1e-6, err
    hs = 1e-6 * pot.sigma
    fds = (L(s.positions, pot.sigma + hs) - L(s.positions, pot.sigma - hs)) / (2 * hs)
    assert abs(out["dsigma"] - fds) <= 1e-6 * abs(fds), (out["dsigma"], fds)
    he = 1e-6 * pot.eps
    fde = (L(s.positions, pot.sigma, pot.eps + he) - L(s.positions, pot.sigma, pot.eps - he)) / (2 * he)
    assert abs(out["deps"] - fde) <= 1e-6 * abs(fde), (out["deps"], fde)
    # The single-precision forms of G against the FP64 form (which the check
    # above pins to central differences): they are limited by G's own rounding,
    # not by the differences.  Measured on a B200: TF32x3 4.6e-6 (positions) and
    # 7.2e-6 (sigma), FP32 1.2e-6 and 2.8e-6 — above the 1e-6 bar, which only
    # the FP64 form (the default) meets; the bounds here sit at about twice those.
    for precision, tol in (("tf32x3", 1e-5), ("fp32", 5e-6)):
        o = mcc3_adjoint_lj(s, pot, calc, phi32, W32, precision=precision)
        e = np.max(np.abs(o["dpos"] - out["dpos"])) / np.max(np.abs(out["dpos"]))
        assert e <= tol, (precision, e)
        assert abs(o["dsigma"] - out["dsigma"]) <= tol * abs(out["dsigma"]), precision

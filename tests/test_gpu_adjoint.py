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


def test_adjoint_at_scale_vs_central_differences(fcb, cuda_device):
    """The 256-atom cell, modes 0..63: the adjoint against central differences
    of L evaluated with the GPU's bit-exact FP64 Ψ and an FP64 contraction on
    the device (h = 2e-3 Å on atoms clear of the LJ truncation; 1e-6 relative
    for σ).  Tolerance 1e-5 of the largest component."""
    import torch
    from fcb200.adjoint import mcc3_adjoint_lj
    from conftest import atoms_clear_of_cutoff
    s = fcc_system((4, 4, 4), 0.05, 1234)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(0.0, AR["r_cut"])
    n, M = 3 * s.n_atoms, 64
    dyn = fcb.dynamical_matrix(s, pot, calc, device="cuda")
    _, _, phi = fcb.get_modes(dyn, 3, phi32=True)
    phi64 = phi[:, :M].double()
    W = torch.from_numpy(np.random.default_rng(9).normal(size=(M, M, M))).to(cuda_device)
    inv_sqrt_m = torch.from_numpy(np.repeat(s.masses, 3) ** -0.5).to(cuda_device)

    def L(sys_, sigma=pot.sigma):
        p = fcb.LJ(sigma, pot.eps, pot.r_cut)
        psi = fcb.third_order(sys_, p, calc, device="cuda").values          # n×n×n column-major FP64
        t = psi.permute(2, 1, 0)                                            # [k][j][i] row-major view
        t = t * inv_sqrt_m[None, None, :] * inv_sqrt_m[None, :, None] * inv_sqrt_m[:, None, None]
        k3 = torch.einsum("kji,ip,jq,ks->pqs", t, phi64, phi64, phi64)
        return float((k3 * W.permute(0, 1, 2)).sum())   # W[p,q,s] against K3[p,q,s]

    W32 = np.asfortranarray(W.cpu().numpy().astype(np.float32))
    phi32 = np.asfortranarray(phi.cpu().numpy())
    out = mcc3_adjoint_lj(s, pot, calc, phi32, W32, precision="tf32x3")
    clear = atoms_clear_of_cutoff(s, AR["r_cut"])
    h = 2e-3
    fd, ad = [], []
    for a, d in [(int(clear[0]), 0), (int(clear[7]), 1), (int(clear[31]), 2), (int(clear[60]), 0)]:
        pp = s.positions.copy()
        pp.reshape(-1, 3)[a, d] += h
        lp = L(fcb.SuperCellSystem(pp, s.masses, s.box_sizes))
        pp.reshape(-1, 3)[a, d] -= 2 * h
        lm = L(fcb.SuperCellSystem(pp, s.masses, s.box_sizes))
        fd.append((lp - lm) / (2 * h))
        ad.append(out["dpos"][a, d])
    scale = np.max(np.abs(out["dpos"]))
    assert np.max(np.abs(np.array(fd) - np.array(ad))) <= 1e-5 * scale
    hs = 1e-6 * pot.sigma
    fds = (L(s, pot.sigma + hs) - L(s, pot.sigma - hs)) / (2 * hs)
    assert abs(fds - out["dsigma"]) <= 1e-5 * abs(fds)
    assert abs(out["deps"] - out["L"] / pot.eps) <= 1e-9 * abs(out["deps"])

"""get_modes on the GPU (fcb200_get_modes, cuSOLVER syevd) vs the host
restatement oracle.get_modes (numpy eigh, restating src/dynmat.jl:123-141).

Eigenvectors are unique only up to sign (and rotation inside degenerate
eigenspaces), so the checks are basis-free:
  * eigenvalues:            max|λ - λ_ref| <= 1e-10 · max|λ_ref|
  * orthonormality:         max|VᵀV - I|   <= 1e-12
  * eigen-equation:         max|D V - V Λ| <= 1e-10 · max|D|  (Λ before rigid zeroing)
  * rigid-mode zeroing:     exactly the reference's rule (stable sortperm of |λ|) applied
                            to the GPU's own eigenvalues, bit for bit
and K3 built from the GPU's FP32 modes matches the FP64 contraction of the same
φ within the mcc3 tolerance (1e-5 normwise).
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu


def _dynmat(fcb, oracle, cells, std, seed):
    s = fcc_system(cells, std, seed)
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    return s, oracle.dynamical_matrix(ifc2, s.masses)


def _rigid_rule(w, k):
    out = np.array(w, copy=True)
    out[np.argsort(np.abs(w), kind="stable")[:k]] = 0.0
    return out


@pytest.mark.parametrize("cells,std,seed", [((2, 2, 2), 0.05, 3), ((4, 4, 4), 0.05, 1234), ((3, 3, 3), 0.0, 0)])
def test_get_modes_vs_lapack(fcb, oracle, cuda_device, cells, std, seed):
    _, D = _dynmat(fcb, oracle, cells, std, seed)
    w_ref, _ = oracle.get_modes(D, 0)
    w_raw, V = fcb.get_modes(D, 0)
    scale = np.max(np.abs(w_ref))
    assert np.max(np.abs(w_raw - w_ref)) <= 1e-10 * scale
    assert np.all(np.diff(w_raw) >= 0)
    n = D.shape[0]
    assert np.max(np.abs(V.T @ V - np.eye(n))) <= 1e-12
    assert np.max(np.abs(D @ V - V * w_raw[None, :])) <= 1e-10 * np.max(np.abs(D))
    w3, V3 = fcb.get_modes(D, 3)
    assert np.array_equal(w3, _rigid_rule(w_raw, 3))
    assert np.array_equal(V3, V)


def test_rigid_zeroing_ties_are_stable(fcb, cuda_device):
    # ascending eigenvalues [-1, -0.5, 0.5, 1, 2]: |λ| ties keep index order
    D = np.diag([1.0, -0.5, 2.0, -1.0, 0.5])
    w2, _ = fcb.get_modes(D, 2)
    assert np.array_equal(w2, np.array([-1.0, 0.0, 0.0, 1.0, 2.0]))
    w3, _ = fcb.get_modes(D, 3)
    assert np.array_equal(w3, np.array([0.0, 0.0, 0.0, 1.0, 2.0]))
    w0, _ = fcb.get_modes(D, 0)
    assert np.array_equal(w0, np.array([-1.0, -0.5, 0.5, 1.0, 2.0]))
    w5, _ = fcb.get_modes(D, 5)
    assert np.array_equal(w5, np.zeros(5))


def test_device_tensors_and_phi32(fcb, oracle, cuda_device):
    import torch
    _, D = _dynmat(fcb, oracle, (2, 2, 2), 0.05, 9)
    w_h, V_h = fcb.get_modes(D, 3)
    Dd = torch.from_numpy(np.asfortranarray(D)).to(cuda_device)
    w_d, V_d, f_d = fcb.get_modes(Dd, 3, phi32=True)
    assert w_d.is_cuda and V_d.is_cuda and f_d.is_cuda and f_d.dtype == torch.float32
    torch.cuda.synchronize()
    # same solver, same input: identical results whether the buffers are host or device
    assert np.array_equal(w_d.cpu().numpy(), w_h)
    assert np.array_equal(V_d.cpu().numpy(), V_h)
    assert np.array_equal(f_d.cpu().numpy(), V_h.astype(np.float32))


def test_in_place(fcb, oracle, cuda_device):
    from fcb200 import _lib
    from fcb200.arrays import ptr
    _, D = _dynmat(fcb, oracle, (2, 2, 2), 0.05, 11)
    w_ref, V_ref = fcb.get_modes(D, 3)
    A = np.asfortranarray(D.copy())
    w = np.empty(A.shape[0])
    _lib.check(_lib.lib().fcb200_get_modes(_lib.handle(0), ptr(A), A.shape[0], 3, ptr(w), ptr(A), 0, 0))
    assert np.array_equal(w, w_ref) and np.array_equal(A, V_ref)


def test_errors(fcb, cuda_device):
    from fcb200 import _lib
    from fcb200.arrays import ptr
    D = np.eye(4)
    w = np.empty(4)
    L, h = _lib.lib(), _lib.handle(0)
    assert L.fcb200_get_modes(h, ptr(D), 4, 5, ptr(w), 0, 0, 0) == _lib.FCB_ERR_ARG
    assert L.fcb200_get_modes(h, ptr(D), 0, 0, ptr(w), 0, 0, 0) == _lib.FCB_ERR_ARG
    assert L.fcb200_get_modes(h, 0, 4, 0, ptr(w), 0, 0, 0) == _lib.FCB_ERR_ARG
    with pytest.raises(ValueError):
        fcb.get_modes(np.zeros((3, 4)))


def test_k3_from_device_modes(fcb, oracle, cuda_device):
    """Device dynamical matrix → device modes → snapshot K3, against the FP64
    contraction of the oracle's Ψ with the same FP32 φ."""
    import torch
    s = fcc_system((2, 2, 2), 0.05, 21)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    dyn = fcb.dynamical_matrix(s, pot, calc, device="cuda")
    _, _, phi = fcb.get_modes(dyn, 3, phi32=True)
    psi, k3 = fcb.snapshot_lj(s, pot, calc, phi, precision="bf16x3")
    torch.cuda.synchronize()
    phi_h = phi.cpu().numpy().astype(np.float64)
    ref_psi = oracle.mass_weight_third_order(
        oracle.third_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12), s.masses)
    ref = oracle.mcc3(ref_psi.astype(np.float32).astype(np.float64), phi_h)
    k = k3.cpu().numpy() if hasattr(k3, "cpu") else np.asarray(k3)
    assert np.max(np.abs(k - ref)) / np.max(np.abs(ref)) <= 1e-5

"""mcc3 on the GPU vs the FP64 contraction oracle (oracle/oracle.py:mcc3,
restating src/mcc.jl:29-51 and :89-134).

Tolerance (stated per the contract): normwise error
    max|K - K_ref| / max|K_ref| <= 1e-5
for FP32, BF16×3 and TF32×3, with K_ref the FP64 contraction of the same FP32
inputs.  RMS relative error is checked too.
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu

TOL = 1e-5
PRECISIONS = ["fp32", "bf16x3", "tf32x3"]


def _inputs(fcb, oracle, cells, std, seed):
    s = fcc_system(cells, std, seed)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    psi = oracle.third_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    psi = oracle.mass_weight_third_order(psi, s.masses).astype(np.float32, order="F")
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    return psi, np.asfortranarray(phi.astype(np.float32))


def _err(k, ref):
    scale = np.max(np.abs(ref))
    d = np.asarray(k, dtype=np.float64) - ref
    return np.max(np.abs(d)) / scale, np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(ref ** 2))


@pytest.fixture(scope="module")
def small(fcb, oracle):
    psi, phi = _inputs(fcb, oracle, (2, 2, 2), 0.05, 31)          # n = 96
    return psi, phi, oracle.mcc3(psi.astype(np.float64), phi.astype(np.float64))


@pytest.fixture(scope="module")
def medium(fcb, oracle):
    psi, phi = _inputs(fcb, oracle, (3, 3, 3), 0.05, 32)          # n = 324 (padded split planes)
    return psi, phi, oracle.mcc3(psi.astype(np.float64), phi.astype(np.float64))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_mcc3_small(fcb, cuda_device, small, precision):
    import torch
    psi, phi, ref = small
    k = fcb.mcc3(torch.from_numpy(psi).cuda(), torch.from_numpy(phi).cuda(), precision=precision)
    mx, rms = _err(k.cpu().numpy(), ref)
    assert mx <= TOL and rms <= TOL, (precision, mx, rms)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_mcc3_medium_padded(fcb, cuda_device, medium, precision):
    import torch
    psi, phi, ref = medium
    k = fcb.mcc3(torch.from_numpy(psi).cuda(), torch.from_numpy(phi).cuda(), precision=precision)
    mx, rms = _err(k.cpu().numpy(), ref)
    assert mx <= TOL and rms <= TOL, (precision, mx, rms)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_mcc3_blocked_host_equals_full(fcb, cuda_device, small, precision):
    import torch
    psi, phi, ref = small
    full = fcb.mcc3(torch.from_numpy(psi).cuda(), torch.from_numpy(phi).cuda(), precision=precision).cpu().numpy()
    blk = fcb.mcc3(psi, phi, 32, precision=precision)      # host result, like mcc.jl:97
    assert isinstance(blk, np.ndarray) and blk.shape == (96, 96, 96)
    mx, _ = _err(blk, ref)
    assert mx <= TOL
    assert np.allclose(blk, full, rtol=0, atol=1e-6 * np.max(np.abs(full)))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_mcc3_mode_windows(fcb, cuda_device, small, precision):
    psi, phi, ref = small
    w = fcb.mcc3_window(psi, phi, (0, 32), (32, 64), (64, 96), precision=precision)
    sub = ref[0:32, 32:64, 64:96]
    d = np.max(np.abs(np.asarray(w, dtype=np.float64) - sub)) / np.max(np.abs(ref))
    assert d <= TOL


def test_mcc3_random_nonsymmetric_inputs(fcb, oracle, cuda_device):
    """General (non-symmetric) Ψ and non-orthogonal φ: catches index-order bugs."""
    import torch
    rng = np.random.default_rng(77)
    n = 40
    psi = np.asfortranarray(rng.normal(size=(n, n, n)).astype(np.float32))
    phi = np.asfortranarray(rng.normal(size=(n, n)).astype(np.float32))
    ref = np.einsum("ijk,in,jm,kl->nml", psi.astype(np.float64), phi.astype(np.float64),
                    phi.astype(np.float64), phi.astype(np.float64))
    for precision in PRECISIONS:
        k = fcb.mcc3(torch.from_numpy(psi).cuda(), torch.from_numpy(phi).cuda(), precision=precision)
        mx, _ = _err(k.cpu().numpy(), ref)
        assert mx <= TOL, (precision, mx)


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3", "fp32"])
def test_snapshot_fused_matches_oracle(fcb, oracle, cuda_device, precision):
    import torch
    s = fcc_system((2, 2, 2), 0.05, 41)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    psi64 = oracle.third_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    mw = oracle.mass_weight_third_order(psi64.copy(order="F"), s.masses)
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    phi32 = np.asfortranarray(phi.astype(np.float32))
    ref = oracle.mcc3(mw, phi32.astype(np.float64))
    from fcb200.arrays import julia_empty
    n = 96
    psi_dev = julia_empty((n, n, n), np.float64, "cuda")
    _, k3 = fcb.snapshot_lj(s, pot, calc, torch.from_numpy(phi32).cuda(), precision=precision, psi_out=psi_dev)
    torch.cuda.synchronize()
    assert np.array_equal(psi_dev.cpu().numpy(), psi64)
    mx, rms = _err(k3.cpu().numpy(), ref)
    assert mx <= TOL and rms <= TOL, (mx, rms)


def test_bad_precision_is_an_error(fcb, cuda_device, small):
    from fcb200 import _lib
    psi, phi, _ = small
    st = _lib.lib().fcb200_mcc3(_lib.handle(0), psi.ctypes.data, phi.ctypes.data, 96, 0, 96, 0, 96, 0, 96, 9,
                                np.empty(96 ** 3, np.float32).ctypes.data, None)
    assert st == _lib.FCB_ERR_ARG

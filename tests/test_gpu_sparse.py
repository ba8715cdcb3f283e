"""Block-sparse first mode product of the LJ snapshot (fcb200_snapshot_lj
with a split precision) vs the FP64 contraction oracle.

mcc3 is defined as the dense contraction (src/mcc.jl:29-51); the block-sparse
form skips only products with structurally zero Ψ entries, so it must give the
same K3 within the mcc3 tolerance:
    max|K - K_ref| / max|K_ref| <= 1e-5,  RMS(K - K_ref)/RMS(K_ref) <= 1e-5,
with K_ref = oracle.mcc3 of the FP32 mass-weighted oracle Ψ and the same φ.
The FP64 Ψ written by the sparse form must stay bit-identical to the oracle.
"""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _case(fcb, oracle, cells, std, seed):
    s = fcc_system(cells, std, seed)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    psi64 = oracle.third_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    psi_mw = oracle.mass_weight_third_order(psi64.copy(order="F"), s.masses).astype(np.float32).astype(np.float64)
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    return s, pot, calc, psi64, psi_mw, np.asfortranarray(phi.astype(np.float32))


def _err(k, ref):
    d = np.asarray(k, dtype=np.float64) - ref
    return np.max(np.abs(d)) / np.max(np.abs(ref)), np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(ref ** 2))


@pytest.fixture(scope="module")
def c324(fcb, oracle):
    return _case(fcb, oracle, (3, 3, 3), 0.05, 17)      # 108 atoms, about 67 per neighbourhood


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_sparse_snapshot_matches_fp64(fcb, oracle, cuda_device, c324, precision):
    s, pot, calc, psi64, psi_mw, phi = c324
    n = 3 * s.n_atoms
    psi_out = np.empty((n, n, n), order="F")
    _, k3 = fcb.snapshot_lj(s, pot, calc, phi, precision=precision, psi_out=psi_out)
    ref = oracle.mcc3(psi_mw, phi.astype(np.float64))
    mx, rms = _err(k3, ref)
    assert mx <= TOL and rms <= TOL, (mx, rms)
    assert np.array_equal(psi_out, psi64)
    # the dense products give the same K3 within the tolerance, by a different rounding path
    _, k3d = fcb.snapshot_lj(s, pot, calc, phi, precision=precision, dense=True)
    assert not np.array_equal(k3, k3d)
    assert _err(k3d, ref)[0] <= TOL


def test_sparse_mode_window_and_device_buffers(fcb, oracle, cuda_device, c324):
    import torch
    s, pot, calc, psi64, psi_mw, phi = c324
    lo, hi = 7, 130
    d_phi = torch.from_numpy(phi).to(cuda_device)
    from fcb200.arrays import julia_empty
    M = hi - lo
    k3 = julia_empty((M, M, M), np.float32, "cuda")
    fcb.snapshot_lj(s, pot, calc, d_phi, precision="bf16x3", modes=(lo, hi), k3_out=k3)
    torch.cuda.synchronize()
    ref = oracle.mcc3(psi_mw, phi.astype(np.float64))[lo:hi, lo:hi, lo:hi]
    mx, rms = _err(k3.cpu().numpy(), ref)
    assert mx <= TOL and rms <= TOL, (mx, rms)


@pytest.fixture(scope="module")
def c768(fcb, oracle):
    case = _case(fcb, oracle, (4, 4, 4), 0.05, 1234)
    return case + (oracle.mcc3(case[4], case[5].astype(np.float64)),)


# 256 atoms take the compact form (neighbourhood-compact first product, grouped
# second product, MN-major third product) in both split precisions.
@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_sparse_snapshot_256_atoms(fcb, oracle, cuda_device, c768, precision):
    s, pot, calc, psi64, psi_mw, phi, ref = c768
    n = 3 * s.n_atoms
    psi_out = np.empty((n, n, n), order="F")
    _, k3 = fcb.snapshot_lj(s, pot, calc, phi, precision=precision, psi_out=psi_out)
    mx, rms = _err(k3, ref)
    assert mx <= TOL and rms <= TOL, (mx, rms)
    assert np.array_equal(psi_out, psi64)


def test_compact_mode_window(fcb, oracle, cuda_device, c768):
    # 304 modes: padded to 512 rows per block, a partial last 256-wide mode tile
    import torch
    from fcb200.arrays import julia_empty
    s, pot, calc, psi64, psi_mw, phi, ref = c768
    lo, hi = 8, 312
    M = hi - lo
    k3 = julia_empty((M, M, M), np.float32, "cuda")
    fcb.snapshot_lj(s, pot, calc, torch.from_numpy(phi).to(cuda_device), precision="bf16x3", modes=(lo, hi),
                    k3_out=k3)
    torch.cuda.synchronize()
    mx, rms = _err(k3.cpu().numpy(), ref[lo:hi, lo:hi, lo:hi])
    assert mx <= TOL and rms <= TOL, (mx, rms)


def test_non_cubic_cell(fcb, oracle, cuda_device):
    s, pot, calc, psi64, psi_mw, phi = _case(fcb, oracle, (3, 4, 3), 0.04, 5)
    _, k3 = fcb.snapshot_lj(s, pot, calc, phi, precision="bf16x3")
    ref = oracle.mcc3(psi_mw, phi.astype(np.float64))
    mx, rms = _err(k3, ref)
    assert mx <= TOL and rms <= TOL, (mx, rms)


def test_every_atom_a_neighbour(fcb, oracle, cuda_device):
    # 2×2×2 with r_cut 8.5 Å: every atom is in every neighbourhood (the sparse
    # form's largest tables relative to the cell)
    s, pot, calc, psi64, psi_mw, phi = _case(fcb, oracle, (2, 2, 2), 0.05, 3)
    _, k3 = fcb.snapshot_lj(s, pot, calc, phi, precision="bf16x3")
    _, k3d = fcb.snapshot_lj(s, pot, calc, phi, precision="bf16x3", dense=True)
    ref = oracle.mcc3(psi_mw, phi.astype(np.float64))
    assert _err(k3, ref)[0] <= TOL and _err(k3d, ref)[0] <= TOL
    assert not np.array_equal(k3, k3d)

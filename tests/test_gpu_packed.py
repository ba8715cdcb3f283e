"""Packed K3 (FCB_K3_PACKED): the symmetry-unique entries K3[p,q,s], p <= q <= s,
at s(s+1)(s+2)/6 + q(q+1)/2 + p.  The compact snapshot form writes them
directly from its third product, the other forms pack a full K3; either way
the packed entries equal the full output's entries at those positions bit for
bit, and the unpacked tensor meets the mcc3 tolerance against the FP64 oracle
(max|ΔK|/max|K| <= 1e-5, RMS likewise)."""
import numpy as np
import pytest

from conftest import AR, fcc_system

pytestmark = pytest.mark.gpu


def _case(fcb, oracle, cells, std, seed):
    s = fcc_system(cells, std, seed)
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    return s, pot, calc, np.asfortranarray(phi.astype(np.float32))


@pytest.mark.parametrize("cells,precision,modes,dense", [
    ((4, 4, 4), "bf16x3", None, False),        # compact form: packed by the third product
    ((4, 4, 4), "tf32x3", (8, 312), False),    # compact form, a mode window of 304 (partial tiles)
    ((3, 3, 3), "bf16x3", None, False),        # dense-layout sparse form: packed afterwards
    ((2, 2, 2), "fp32", None, False),          # dense FP32 products
    ((2, 2, 2), "bf16x3", None, True),         # dense split products
])
def test_packed_equals_full(fcb, oracle, cuda_device, cells, precision, modes, dense):
    import torch
    from fcb200.mcc import packed_k3_index
    s, pot, calc, phi = _case(fcb, oracle, cells, 0.05, 7)
    d_phi = torch.from_numpy(phi).to(cuda_device)
    _, full = fcb.snapshot_lj(s, pot, calc, d_phi, precision=precision, modes=modes, dense=dense)
    _, packed = fcb.snapshot_lj(s, pot, calc, d_phi, precision=precision, modes=modes, dense=dense, packed=True)
    torch.cuda.synchronize()
    n = 3 * s.n_atoms
    M = n if modes is None else modes[1] - modes[0]
    assert packed.numel() == fcb.packed_k3_count(M)
    idx = torch.from_numpy(packed_k3_index(M)).to(cuda_device)
    flat = full.permute(2, 1, 0).reshape(-1)          # column-major memory order
    assert torch.equal(flat[idx], packed)


def test_packed_host_output_vs_oracle(fcb, oracle, cuda_device):
    s, pot, calc, phi = _case(fcb, oracle, (4, 4, 4), 0.05, 1234)
    psi = oracle.third_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 1e-12)
    mw = oracle.mass_weight_third_order(psi, s.masses).astype(np.float32).astype(np.float64)
    del psi
    ref = oracle.mcc3(mw, phi.astype(np.float64))
    n = 3 * s.n_atoms
    out = np.empty(fcb.packed_k3_count(n), dtype=np.float32)     # host buffer
    _, k = fcb.snapshot_lj(s, pot, calc, phi, precision="bf16x3", k3_out=out, packed=True)
    full = fcb.unpack_k3(k, n)
    d = full.astype(np.float64) - ref
    assert np.max(np.abs(d)) <= 1e-5 * np.max(np.abs(ref))
    assert np.sqrt(np.mean(d ** 2)) <= 1e-5 * np.sqrt(np.mean(ref ** 2))


def test_packed_sw_snapshot(fcb, oracle, cuda_device):
    import torch
    from fcb200.mcc import packed_k3_index
    s = fcb.displaced(fcb.Diamond(5.43, "Si", (2, 2, 2)), 0.03, 11)
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.AutoDiffCalculator(1e-12, pot.r_cut)
    ifc2 = oracle.second_order_sw(s.positions, s.box_sizes, pot.r_cut, 1e-12)
    _, phi = oracle.get_modes(oracle.dynamical_matrix(ifc2, s.masses))
    d_phi = torch.from_numpy(np.asfortranarray(phi.astype(np.float32))).to(cuda_device)
    _, full = fcb.snapshot_lj(s, pot, calc, d_phi, precision="bf16x3")
    _, packed = fcb.snapshot_lj(s, pot, calc, d_phi, precision="bf16x3", packed=True)
    torch.cuda.synchronize()
    idx = torch.from_numpy(packed_k3_index(3 * s.n_atoms)).to(cuda_device)
    assert torch.equal(full.permute(2, 1, 0).reshape(-1)[idx], packed)

"""Stillinger-Weber IFC2/IFC3 on the GPU vs the oracle and the reference golden
fixtures.  Tolerance: max |Ψ_gpu − Ψ_ref| <= 1e-12 elementwise (eV/Å³), the
north-star bar for matching the reference AutoDiffCalculator."""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sw_diamond_*.npz")))


def _sys(fcb, cells, std, seed):
    s = fcb.Diamond(5.43, "Si", cells)
    return fcb.displaced(s, std, seed) if std > 0 else s


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
def test_sw_third_order_vs_reference_golden(fcb, cuda_device, path):
    d = np.load(path)
    s = fcb.SuperCellSystem(d["positions"], np.full(len(d["positions"]), 28.0855), d["box"])
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.AutoDiffCalculator(float(d["tol"]), pot.r_cut)
    got = fcb.third_order(s, pot, calc, device="cuda").values.cpu().numpy()
    n = int(d["n"])
    ref = np.zeros(n ** 3)
    ref[d["ifc3_index"]] = d["ifc3_value"]
    assert np.max(np.abs(got - ref.reshape((n, n, n), order="F"))) <= TOL
    ifc2 = fcb.second_order(s, pot, calc).values
    assert np.max(np.abs(ifc2 - d["ifc2"])) <= TOL


@pytest.mark.parametrize("cells,std,seed", [((1, 1, 1), 0.0, 0), ((2, 2, 2), 0.03, 3), ((3, 3, 3), 0.03, 4)])
def test_sw_third_order_vs_oracle(fcb, oracle, cuda_device, cells, std, seed):
    s = _sys(fcb, cells, std, seed)
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.AutoDiffCalculator(1e-12, pot.r_cut)
    ref = oracle.third_order_sw(s.positions, s.box_sizes, pot.r_cut, 1e-12)
    got = fcb.third_order(s, pot, calc, device="cuda").values.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= TOL
    # every structural zero of the reference is an exact zero here
    assert np.array_equal(got == 0.0, ref == 0.0)
    ref2 = oracle.second_order_sw(s.positions, s.box_sizes, pot.r_cut, 1e-12)
    got2 = fcb.second_order(s, pot, calc).values
    assert np.max(np.abs(got2 - ref2)) <= TOL


def test_sw_mass_weighted_outputs(fcb, oracle, cuda_device):
    import torch
    from fcb200.arrays import julia_empty
    s = _sys(fcb, (2, 2, 2), 0.03, 9)
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.AutoDiffCalculator(1e-12, pot.r_cut)
    ref = oracle.third_order_sw(s.positions, s.box_sizes, pot.r_cut, 1e-12)
    mw = oracle.mass_weight_third_order(ref.copy(order="F"), s.masses)
    n = 3 * s.n_atoms
    psi = julia_empty((n, n, n), np.float64, "cuda")
    psi32 = julia_empty((n, n, n), np.float32, "cuda")
    fcb.third_order_(psi, s, pot, calc, mass_weighted=True, psi32_mw=psi32)
    torch.cuda.synchronize()
    assert np.max(np.abs(psi.cpu().numpy() - mw)) <= TOL
    assert np.max(np.abs(psi32.cpu().numpy() - mw.astype(np.float32))) <= 1e-6 * np.max(np.abs(mw))
    dyn = fcb.dynamical_matrix(s, pot, calc).values
    ref2 = oracle.dynamical_matrix(oracle.second_order_sw(s.positions, s.box_sizes, pot.r_cut, 1e-12), s.masses)
    assert np.max(np.abs(dyn - ref2)) <= TOL


def test_sw_cutoff_error(fcb, cuda_device):
    s = _sys(fcb, (1, 1, 1), 0.0, 0)
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.AutoDiffCalculator(1e-12, pot.r_cut + 0.1)
    with pytest.raises(AssertionError):
        fcb.third_order(s, pot, calc, device="cuda")

"""Finite-difference force constants on the GPU (fcb200_fd_*).

1. Against the oracle's restatement of the reference (oracle/fd_oracle.c:
   whole-cell energy_loop totals in the reference's loop order, the stencils of
   third_order_FD.jl:43-113 and second_order_FD.jl:3-79 + ASR): the GPU sums
   only the terms that involve the displaced atoms, so the two differ by the
   rounding of the reference's whole-cell cancellation —
   |FD_gpu - FD_oracle| <= 1e-6 + 1e-6·|FD_oracle|.
2. As the independent check it exists for: FD vs the analytical LJ and the
   AD-equivalent SW force constants from the GPU assemblies, within the O(h²)
   truncation of the default step (0.04 bohr): 2e-3 of the largest entry.
Cells keep r_cut below half the box, where the single-minimum-image energy is
smooth (a smaller cell puts stencil points across the image boundary, for the
reference as much as here).
"""
import numpy as np
import pytest

from conftest import AR, atoms_clear_of_cutoff, fcc_system

pytestmark = pytest.mark.gpu

H = 0.04 * 0.5291772109


def _lj_elements(s, rng, count):
    """Two-same (i,α,j,β,i,α) for neighbours j of i, all-same, all-different, and
    two arrangements without a reference stencil."""
    pos, box, N = s.positions.reshape(-1, 3), s.box_sizes, s.n_atoms
    clear = atoms_clear_of_cutoff(s, AR["r_cut"])
    out = []
    while len(out) < 3 * count:
        i = int(rng.choice(clear))
        d = pos - pos[i]
        d -= box * np.round(d / box)
        dist = np.linalg.norm(d, axis=1)
        nb = np.intersect1d(np.nonzero((dist > 0) & (dist < 6.0))[0], clear)
        if nb.size < 2:
            continue
        j, k = (int(x) for x in rng.choice(nb, 2, replace=False))
        a, b, c = (int(x) for x in rng.integers(3, size=3))
        out += [[i, a, j, b, i, a], [i, a, i, a, i, a], [i, a, j, b, k, c]]
    out += [[0, 0, 0, 1, 5, 2], [0, 0, 5, 1, 5, 2]]
    return np.array(out, dtype=np.int64)


def _analytic(psi, e):
    i, a, j, b, k, c = e
    if i == j == k:
        return psi[3 * i + a, 3 * i + a, 3 * i + a]
    if i == k != j:
        return psi[3 * i + a, 3 * j + b, 3 * i + a]     # the reference's stencil ignores γ
    return psi[3 * i + a, 3 * j + b, 3 * k + c]


@pytest.fixture(scope="module")
def lj256(fcb):
    return fcc_system((4, 4, 4), 0.05, 1234)


def test_fd_third_lj_vs_oracle_and_analytic(fcb, oracle, cuda_device, lj256):
    s = lj256
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    el = _lj_elements(s, np.random.default_rng(4), 12)
    gpu = fcb.third_order_fd(s, pot, el, H)
    ref = oracle.fd_third_order("lj", s.positions, s.box_sizes, el, H, pot.sigma, pot.eps, pot.r_cut)
    assert np.array_equal(np.isnan(gpu), np.isnan(ref))
    assert np.isnan(gpu[-1]) and np.isnan(gpu[-2])
    ok = ~np.isnan(ref)
    assert np.all(np.abs(gpu[ok] - ref[ok]) <= 1e-6 + 1e-6 * np.abs(ref[ok]))
    psi = oracle.third_order_lj(s.positions, s.box_sizes, pot.sigma, pot.eps, pot.r_cut, 0.0)
    ana = np.array([_analytic(psi, e) for e in el[ok]])
    assert np.max(np.abs(gpu[ok] - ana)) <= 2e-3 * np.max(np.abs(psi))


def test_fd_single_element_api(fcb, cuda_device, lj256):
    s = lj256
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    v = fcb.third_order_finite_diff_eng(s, pot, [1, 2, 1], [1, 3, 1])       # 1-based, two-same
    assert v == fcb.third_order_fd(s, pot, [[0, 0, 1, 2, 0, 0]])[0]
    with pytest.warns(UserWarning):
        assert fcb.third_order_finite_diff_eng(s, pot, [1, 1, 2], [1, 2, 3]) is None
    with pytest.raises(AssertionError):
        fcb.third_order_finite_diff_eng(s, pot, [1, 2, s.n_atoms + 1], [1, 1, 1])
    with pytest.raises(AssertionError):
        fcb.third_order_finite_diff_eng(s, pot, [1, 2, 3], [1, 4, 1])


def test_fd_third_sw_vs_oracle_and_ad(fcb, oracle, cuda_device):
    s = fcb.displaced(fcb.Diamond(5.43, "Si", (2, 2, 2)), 0.03, 11)
    pot = fcb.StillingerWeberSilicon()
    pos, box, N = s.positions.reshape(-1, 3), s.box_sizes, s.n_atoms
    rng = np.random.default_rng(2)
    el = []
    for _ in range(10):
        i = int(rng.integers(N))
        d = pos - pos[i]
        d -= box * np.round(d / box)
        nb = np.nonzero((np.linalg.norm(d, axis=1) > 0) & (np.linalg.norm(d, axis=1) < 3.0))[0]
        j, k = (int(x) for x in rng.choice(nb, 2, replace=False))
        a, b, c = (int(x) for x in rng.integers(3, size=3))
        el += [[i, a, j, b, k, c], [j, a, i, b, k, c], [i, a, j, b, i, a], [i, b, i, b, i, b]]
    el = np.array(el, dtype=np.int64)
    gpu = fcb.third_order_fd(s, pot, el, H)
    ref = oracle.fd_third_order("sw", s.positions, s.box_sizes, el, H)
    assert np.all(np.abs(gpu - ref) <= 1e-6 + 1e-6 * np.abs(ref))
    calc = fcb.AutoDiffCalculator(0.0, pot.r_cut)
    psi = fcb.third_order(s, pot, calc).values
    ana = np.array([_analytic(psi, e) for e in el])
    assert np.max(np.abs(gpu - ana)) <= 2e-3 * np.max(np.abs(psi))


def test_fd_second_order_lj(fcb, oracle, cuda_device):
    # oracle-sized case: 2×2×2 with a 4.5 Å cutoff (below half the 10.49 Å box)
    s = fcc_system((2, 2, 2), 0.04, 8)
    pot = fcb.LJ(AR["sigma"], AR["eps"], 4.5)
    calc = fcb.FiniteDiffCalculator(0.0, 4.5)
    gpu = np.asarray(fcb.second_order(s, pot, calc).values)
    ref = oracle.fd_second_order("lj", s.positions, s.box_sizes, 4.5, H, pot.sigma, pot.eps, pot.r_cut)
    assert np.max(np.abs(gpu - ref)) <= 1e-6 * max(1.0, np.max(np.abs(ref)))
    # off-diagonal blocks are filled symmetrically; the ASR diagonal blocks sum
    # different stencils, so they are symmetric only to the truncation error
    assert np.max(np.abs(gpu - gpu.T)) <= 2e-3 * np.max(np.abs(gpu))
    # Full cell vs the analytical IFC2.  The LJ energy is truncated, not shifted,
    # at r_cut: a stencil whose pair crosses r_cut sees the energy jump, so the
    # comparison takes the off-diagonal blocks of pairs at least 0.2 Å inside
    # the cutoff (the ASR diagonal blocks sum over every pair).
    s4 = fcc_system((4, 4, 4), 0.05, 1234)
    pot4 = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    fd = np.asarray(fcb.second_order(s4, pot4, fcb.FiniteDiffCalculator(0.0, AR["r_cut"])).values)
    ana = np.asarray(fcb.second_order(s4, pot4, fcb.AnalyticalCalculator(0.0, AR["r_cut"])).values)
    p = s4.positions.reshape(-1, 3)
    d = p[:, None, :] - p[None, :, :]
    d -= s4.box_sizes * np.round(d / s4.box_sizes)
    dist = np.linalg.norm(d, axis=2)
    keep = (dist > 0) & (dist < AR["r_cut"] - 0.2)
    mask = np.repeat(np.repeat(keep, 3, axis=0), 3, axis=1)
    assert np.max(np.abs(fd - ana)[mask]) <= 2e-3 * np.max(np.abs(ana))


def test_fd_second_order_sw(fcb, oracle, cuda_device):
    s = fcb.displaced(fcb.Diamond(5.43, "Si", (2, 2, 2)), 0.03, 12)
    pot = fcb.StillingerWeberSilicon()
    calc = fcb.FiniteDiffCalculator(1e-12, pot.r_cut)
    gpu = np.asarray(fcb.second_order(s, pot, calc).values)
    ref = oracle.fd_second_order("sw", s.positions, s.box_sizes, pot.r_cut, H)
    ref[np.abs(ref) < 1e-12] = 0.0
    assert np.max(np.abs(gpu - ref)) <= 1e-6 * max(1.0, np.max(np.abs(ref)))
    # Against the AD IFC2 the pair list must reach the second neighbours that a
    # three-body term couples (up to twice the SW cutoff); the reference's FD
    # calculator with r_cut = the SW cutoff leaves those entries zero.
    fd2 = np.asarray(fcb.second_order(s, pot, fcb.FiniteDiffCalculator(1e-12, 2 * pot.r_cut)).values)
    ad = np.asarray(fcb.second_order(s, pot, fcb.AutoDiffCalculator(1e-12, pot.r_cut)).values)
    assert np.max(np.abs(fd2 - ad)) <= 2e-3 * np.max(np.abs(ad))


def test_fd_errors(fcb, cuda_device):
    from fcb200 import _lib
    s = fcc_system((2, 2, 2), 0.0, 0)
    pot = fcb.LJ(AR["sigma"], AR["eps"], 4.5)
    with pytest.raises(AssertionError):
        fcb.third_order_fd(s, pot, [[0, 0, 1, 1, 40, 0]])
    L = _lib.lib()
    out = np.empty(1)
    assert L.fcb200_fd_third_order_lj(_lib.handle(0), s.positions.ctypes.data, s.n_atoms, s.box_sizes.ctypes.data,
                                      3.4, 0.24, 4.5, np.zeros(6, np.int64).ctypes.data, 1, -1.0,
                                      out.ctypes.data, 0) == _lib.FCB_ERR_ARG

"""The column-slab form of the LJ oracle (oracle_third_order_lj_slab) and the
windowed FP64 contraction built on it, which check the 400-atom cell without
holding its 13.8 GB dense Ψ: every slab equals the same columns of the full
oracle tensor bit for bit, the slab mass weighting equals
mass_weight_third_order entry for entry, and the windowed K3 equals the full
FP64 contraction (to FP64 rounding)."""
import numpy as np

from conftest import AR, fcc_system


def test_slabs_equal_full_oracle(oracle):
    s = fcc_system((3, 3, 3), 0.05, 17)
    m = np.linspace(30.0, 50.0, s.n_atoms)
    full = oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    mw = oracle.mass_weight_third_order(full.copy(order="F"), m)
    seen = 0
    for j0, j1, slab in oracle.lj_slabs(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12,
                                        atoms_per_slab=7):
        assert np.array_equal(slab, full[:, j0:j1, :])
        assert np.array_equal(oracle.mass_weight_slab(slab, m, j0), mw[:, j0:j1, :])
        seen += j1 - j0
    assert seen == 3 * s.n_atoms


def test_windowed_contraction_equals_full(oracle):
    s = fcc_system((3, 3, 3), 0.05, 17)
    m = np.linspace(30.0, 50.0, s.n_atoms)
    full = oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    mw32 = oracle.mass_weight_third_order(full, m).astype(np.float32).astype(np.float64)
    phi = np.linalg.qr(np.random.default_rng(3).normal(size=(324, 324)))[0].astype(np.float32).astype(np.float64)
    ref = oracle.mcc3(mw32, phi)
    P, Q, S = np.arange(0, 40), np.arange(100, 130), np.arange(300, 324)
    got = oracle.mcc3_windows_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12, m, phi,
                                 [(P, Q, S), (S, P, Q)])
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got[0] - ref[np.ix_(P, Q, S)])) <= 1e-13 * scale
    assert np.max(np.abs(got[1] - ref[np.ix_(S, P, Q)])) <= 1e-13 * scale

"""Host-side logic of the Python mirror (no GPU needed)."""
import numpy as np
import pytest

from conftest import AR, fcc_system


def test_fcc_ordering_matches_reference_golden_layout(fcb):
    s = fcb.FCC(AR["a"], "Ar", (4, 4, 4))
    assert s.n_atoms == 256
    assert np.allclose(s.positions[0], 0.0)
    # Atom 2 sits at (a/2, a/2, 0): the layout the reference's golden values imply.
    assert np.allclose(s.positions[1], [AR["a"] / 2, AR["a"] / 2, 0.0])
    assert np.allclose(s.box_sizes, 4 * AR["a"])
    assert np.allclose(s.masses, 39.95)


def test_diamond_builder(fcb):
    s = fcb.Diamond(5.43, "Si", (3, 3, 3))
    assert s.n_atoms == 216
    d = s.positions[:, None, :] - s.positions[None, :, :]
    d -= np.round(d / s.box_sizes) * s.box_sizes
    r = np.sqrt((d ** 2).sum(-1))
    nn = np.sort(r, axis=1)[:, 1:5]
    assert np.allclose(nn, 5.43 * np.sqrt(3) / 4)


def test_displacement_is_seeded(fcb):
    a = fcb.displaced(fcc_system((2, 2, 2)), 0.05, seed=7)
    b = fcb.displaced(fcc_system((2, 2, 2)), 0.05, seed=7)
    assert np.array_equal(a.positions, b.positions)


def test_cutoff_assertion_before_any_device_work(fcb):
    s = fcc_system((1, 1, 1))
    calc = fcb.AnalyticalCalculator(1e-12, AR["r_cut"])
    pot = fcb.LJ(AR["sigma"], AR["eps"], AR["r_cut"])
    psi = np.zeros((12, 12, 12), order="F")
    with pytest.raises(AssertionError, match="Cutoff"):
        fcb.third_order_(psi, s, pot, calc)
    # third_order_analytical.jl:7 asserts on the potential's cutoff, even when
    # the calculator's is shorter
    s2 = fcc_system((2, 2, 2))
    psi2 = np.zeros((96, 96, 96), order="F")
    with pytest.raises(AssertionError, match="Cutoff"):
        fcb.third_order_(psi2, s2, fcb.LJ(AR["sigma"], AR["eps"], 11.0), calc)
    # second_order_AD.jl:4: the AutoDiffCalculator's cutoff may not exceed the potential's
    with pytest.raises(AssertionError, match="Calculator r_cut"):
        fcb.second_order_(np.zeros((96, 96), order="F"), s2, fcb.LJ(AR["sigma"], AR["eps"], 8.0),
                          fcb.AutoDiffCalculator(1e-12, AR["r_cut"]))


def test_julia_layout_helpers(fcb):
    import torch
    from fcb200.arrays import as_julia, julia_empty
    x = torch.arange(24, dtype=torch.float32).reshape(2, 3, 4)
    j = as_julia(x, np.float32)
    assert j.stride() == (1, 2, 6)
    assert torch.equal(j, x)
    e = julia_empty((3, 4, 5), np.float64, "cpu")
    assert e.flags.f_contiguous
    a = np.arange(24.0).reshape(2, 3, 4)
    assert as_julia(a, np.float64).flags.f_contiguous


def test_block_size_assertion(fcb):
    psi = np.zeros((6, 6, 6), dtype=np.float32, order="F")
    phi = np.eye(6, dtype=np.float32)
    with pytest.raises(AssertionError):
        fcb.mcc3(psi, phi, 4)


def test_asr_checker_quirk(fcb):
    # asr.jl:50 tests `s > tol` without abs: a negative sum passes.
    ifc2 = np.zeros((3, 3))
    ifc2[0, 0] = -1.0
    assert fcb.asr_satisfied(ifc2, 1, 3, 1e-8)
    ifc2[0, 0] = 1.0
    assert not fcb.asr_satisfied(ifc2, 1, 3, 1e-8)


def test_packed_k3_layout_roundtrip(fcb):
    """The packed K3 layout (entry (p,q,s), p <= q <= s, at
    s(s+1)(s+2)/6 + q(q+1)/2 + p) and its unpacking on the host."""
    from fcb200.mcc import packed_k3_index
    for M in (1, 3, 8, 13):
        a = np.random.default_rng(M).normal(size=(M, M, M))
        k = sum(a.transpose(t) for t in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)))
        k = np.asfortranarray(k.astype(np.float32))
        idx = packed_k3_index(M)
        assert idx.shape[0] == fcb.packed_k3_count(M) == len(set(idx.tolist()))
        p, q, s = idx % M, (idx // M) % M, idx // (M * M)
        assert np.all(p <= q) and np.all(q <= s)
        assert np.array_equal(s * (s + 1) * (s + 2) // 6 + q * (q + 1) // 2 + p, np.arange(idx.shape[0]))
        assert np.array_equal(fcb.unpack_k3(k.reshape(-1, order="F")[idx], M), k)


def test_full_symmetry_store_rules_cover_k3_once():
    """The third product's full-symmetry schedule: row tiles (a, b) with
    T(a) <= T(b) (T(x) = x // tile) over every column s, each computed entry
    stored at (a,b,s), at (a,s,b) when T(s) < T(a), at (s,a,b) when
    T(s) > T(b), at (s,b,a) when T(s) > T(b) > T(a) — every entry of the
    M³ output exactly once, for tile widths that divide M or not."""
    for M, tile in ((11, 4), (12, 4), (9, 3), (7, 8), (13, 5), (10, 256)):
        t = lambda x: x // tile
        seen = {}
        for a in range(M):
            for b in range(M):
                if t(a) > t(b):
                    continue
                for s in range(M):
                    ta, tb, ts = t(a), t(b), t(s)
                    outs = [(a, b, s)]
                    if ts < ta:
                        outs.append((a, s, b))
                    if ts > tb:
                        outs.append((s, a, b))
                    if ts > tb > ta:
                        outs.append((s, b, a))
                    for o in outs:
                        seen[o] = seen.get(o, 0) + 1
        assert len(seen) == M ** 3 and set(seen.values()) == {1}, (M, tile)

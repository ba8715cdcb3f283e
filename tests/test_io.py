"""Wire formats (fcb200.io) against the reference's io.jl: parse_xyz
(io.jl:319-353) and save_third_order / save_second_order text output
(io.jl:9-68) — header, 1-based fields, loop order, and a bit-exact read-back.
CPU only."""
import numpy as np
import pytest

from conftest import AR


def test_julia_float_form(fcb):
    from fcb200.io import julia_float
    assert julia_float(1e-5) == "1.0e-5"
    assert julia_float(-2.5e-7) == "-2.5e-7"
    assert julia_float(0.0001) == "0.0001"
    assert julia_float(1e16) == "1.0e16"
    assert julia_float(123.0) == "123.0"
    for x in np.random.default_rng(0).normal(size=200) * 10.0 ** np.random.default_rng(1).integers(-12, 12, 200):
        assert float(julia_float(x)) == x


def test_parse_xyz(fcb, tmp_path):
    rng = np.random.default_rng(3)
    n_atoms, steps = 5, 3
    frames = [rng.normal(size=(n_atoms, 3)) * 4 for _ in range(steps)]
    p = tmp_path / "traj.xyz"
    with open(p, "w") as f:
        for s, fr in enumerate(frames):
            f.write(f"{n_atoms}\nAtoms. Timestep: {s * 10}\n")
            for a, x in enumerate(fr):
                f.write(f"{a + 1} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}\n")
    pos, ids = fcb.parse_xyz(str(p), n_atoms, steps)
    assert len(pos) == steps and len(ids) == steps
    for s in range(steps):
        assert np.array_equal(pos[s], frames[s])
        assert list(ids[s]) == [1, 2, 3, 4, 5]
    # asking for more frames than the file holds leaves the extra ones empty
    pos2, ids2 = fcb.parse_xyz(str(p), n_atoms, steps + 2)
    assert pos2[-1].shape == (0, 3) and ids2[-1].shape == (0,)
    # a frame of the trajectory is a snapshot the library takes as positions
    assert pos[1].reshape(-1).shape == (3 * n_atoms,)


def _small_psi(oracle):
    import fcb200 as fcb
    s = fcb.displaced(fcb.FCC(AR["a"], "Ar", (2, 2, 2)), 0.04, 9)
    return s, oracle.third_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)


def test_save_third_order_txt(fcb, oracle, tmp_path):
    s, psi = _small_psi(oracle)
    N = s.n_atoms
    fc = fcb.DenseForceConstants(psi, "kcal mol^-1 Å^-3", 1e-12)
    path = fcb.save_third_order(fc, N, 3, str(tmp_path))
    lines = open(path).read().splitlines()
    assert lines[0].startswith(f"#{N} atoms, Sum Ψ = ") and lines[0].endswith("Units: kcal mol^-1 Å^-3")
    body = [ln.split() for ln in lines[1:]]
    assert len(body) == np.count_nonzero(psi)
    keys = [tuple(int(x) for x in b[:6]) for b in body]
    # loop order i, j, k, α, β, γ with γ fastest
    assert keys == sorted(keys, key=lambda t: (t[0], t[2], t[4], t[1], t[3], t[5]))
    i, a, j, b, k, c = keys[0]
    assert float(body[0][6]) == psi[3 * (i - 1) + a - 1, 3 * (j - 1) + b - 1, 3 * (k - 1) + c - 1]
    back = fcb.load_third_order_txt(path, N)
    assert np.array_equal(back, psi)


def test_save_second_order_txt_and_npz(fcb, oracle, tmp_path):
    import fcb200 as f
    s = f.displaced(f.FCC(AR["a"], "Ar", (2, 2, 2)), 0.04, 9)
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    path = fcb.save_second_order(ifc2, s.n_atoms, 3, str(tmp_path))
    rows = np.loadtxt(path, comments="#")
    assert rows.shape[0] == np.count_nonzero(ifc2)
    got = np.zeros_like(ifc2)
    got[3 * (rows[:, 0].astype(int) - 1) + rows[:, 1].astype(int) - 1,
        3 * (rows[:, 2].astype(int) - 1) + rows[:, 3].astype(int) - 1] = rows[:, 4]
    assert np.array_equal(got, ifc2)
    p2 = fcb.save_second_order(ifc2, s.n_atoms, 3, str(tmp_path), fmt="npz")
    z = np.load(p2)
    assert np.array_equal(z["F2"], ifc2) and int(z["N_atoms"]) == s.n_atoms and int(z["dimension"]) == 3


def test_formats_and_shapes_checked(fcb, oracle, tmp_path):
    s, psi = _small_psi(oracle)
    with pytest.raises(ValueError):
        fcb.save_third_order(psi, s.n_atoms, 3, str(tmp_path), fmt="JLD2")
    with pytest.raises(AssertionError):
        fcb.save_third_order(psi, s.n_atoms + 1, 3, str(tmp_path))
    p = fcb.save_third_order(psi, s.n_atoms, 3, str(tmp_path), fmt="npz")
    z = np.load(p)
    assert np.array_equal(z["F3"], psi)

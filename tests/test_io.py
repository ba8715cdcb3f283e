"""Wire formats (fcb200.io) against the reference's io.jl: parse_xyz
(io.jl:319-353) and save_third_order / save_second_order text output
(io.jl:9-68) — header, 1-based fields, loop order, and a bit-exact read-back —
and the default JLD2 (HDF5) output: the checksum against its published test
vectors, the reader against a file written by the HDF5 library, the writer's
encodings against that file's, and bit-exact read-back.  CPU only."""
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
    # fewer frames than the file holds: the reference's push! into frame
    # n_steps + 1 is a BoundsError
    with pytest.raises(IndexError):
        fcb.parse_xyz(str(p), n_atoms, steps - 1)
    # blank lines are skipped (readdlm) and a truncated last frame keeps the
    # atoms it has
    q = tmp_path / "cut.xyz"
    with open(q, "w") as f:
        f.write(f"{n_atoms}\nstep 0\n\n")
        for a, x in enumerate(frames[0]):
            f.write(f"{a + 1} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}\n")
        f.write(f"{n_atoms}\nstep 1\n")
        for a, x in enumerate(frames[1][:2]):
            f.write(f"{a + 1} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}\n")
    pos3, ids3 = fcb.parse_xyz(str(q), n_atoms, 2)
    assert np.array_equal(pos3[0], frames[0]) and np.array_equal(pos3[1], frames[1][:2])
    assert list(ids3[1]) == [1, 2]
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
    path = fcb.save_third_order(fc, N, 3, str(tmp_path), fmt="txt")
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
    path = fcb.save_second_order(ifc2, s.n_atoms, 3, str(tmp_path), fmt="txt")
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
        fcb.save_third_order(psi, s.n_atoms, 3, str(tmp_path), fmt="hdf5")
    with pytest.raises(AssertionError):
        fcb.save_third_order(psi, s.n_atoms + 1, 3, str(tmp_path))
    p = fcb.save_third_order(psi, s.n_atoms, 3, str(tmp_path), fmt="npz")
    z = np.load(p)
    assert np.array_equal(z["F3"], psi)


# ---------------------------------------------------------------------------
# JLD2 / HDF5

def test_lookup3_published_vectors(fcb):
    # the test values of Bob Jenkins' lookup3.c (hashlittle)
    from fcb200.hdf5 import lookup3
    assert lookup3(b"", 0) == 0xDEADBEEF
    assert lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert lookup3(b"Four score and seven years ago", 0) == 0x17770551
    assert lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def _hdf5_library_file():
    """A MAT 7.3 file (HDF5, written by the HDF5 library under MATLAB 7.4) from
    scipy's test data, and the MAT 5 file holding the same variable."""
    import os
    scipy_io = pytest.importorskip("scipy.io")
    data = os.path.join(os.path.dirname(scipy_io.matlab.__file__), "tests", "data")
    h5, v5 = os.path.join(data, "testhdf5_7.4_GLNX86.mat"), os.path.join(data, "testdouble_7.4_GLNX86.mat")
    if not (os.path.exists(h5) and os.path.exists(v5)):
        pytest.skip("scipy's MAT test files are not installed")
    return h5, v5


def test_reader_on_a_file_written_by_the_hdf5_library(fcb):
    # superblock 0 after a 512-byte user block, a symbol-table root group
    # (B-tree, symbol-table node, local heap), version-1 object headers and a
    # contiguous layout; the values must equal scipy's reading of the MAT 5
    # file that holds the same variable
    import scipy.io as sio
    h5, v5 = _hdf5_library_file()
    got = fcb.load_force_constants(h5)
    ref = sio.loadmat(v5)["testdouble"]
    assert set(got) == {"testdouble"}
    assert got["testdouble"].shape == ref.shape == (1, 9)
    assert np.array_equal(got["testdouble"], ref)


def test_writer_encodings_match_the_hdf5_library(fcb, tmp_path):
    # the float64 datatype message the writer emits is byte for byte the one
    # the HDF5 library wrote for a MATLAB double
    from fcb200 import hdf5
    h5, _ = _hdf5_library_file()
    lib = hdf5._File(open(h5, "rb").read())
    addr = lib.links(lib.root)["testdouble"]
    lib_dtype = [b for t, b in lib.messages(addr) if t == 0x03][0]
    p = str(tmp_path / "x.jld2")
    hdf5.write(p, {"x": np.zeros((2, 3))})
    ours = hdf5._File(open(p, "rb").read())
    our_dtype = [b for t, b in ours.messages(ours.links(ours.root)["x"]) if t == 0x03][0]
    assert bytes(our_dtype) == bytes(lib_dtype[:len(our_dtype)])


def test_save_third_order_jld2_default(fcb, oracle, tmp_path):
    # the reference's default: jldsave(F3 = values, N_atoms, dimension, unit)
    s, psi = _small_psi(oracle)
    fc = fcb.DenseForceConstants(psi, "kcal mol^-1 Å^-3", 1e-12)
    path = fcb.save_third_order(fc, s.n_atoms, 3, str(tmp_path))
    assert path.endswith("third_order.jld2")
    raw = open(path, "rb").read()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n" and raw[8] == 2          # superblock version 2
    got = fcb.load_force_constants(path)
    assert set(got) == {"F3", "N_atoms", "dimension", "unit"}
    assert got["F3"].shape == psi.shape and np.array_equal(got["F3"], psi)
    assert got["N_atoms"] == s.n_atoms and got["dimension"] == 3
    assert got["unit"] == "kcal mol^-1 Å^-3"
    # every checksum is verified by the reader: a flipped byte in the root
    # group header is reported
    bad = bytearray(raw)
    bad[60] ^= 0xFF
    p2 = str(tmp_path / "bad.jld2")
    open(p2, "wb").write(bytes(bad))
    with pytest.raises(ValueError):
        fcb.load_force_constants(p2)


def test_save_second_order_jld2(fcb, oracle, tmp_path):
    import fcb200 as f
    s = f.displaced(f.FCC(AR["a"], "Ar", (2, 2, 2)), 0.04, 9)
    ifc2 = oracle.second_order_lj(s.positions, s.box_sizes, AR["sigma"], AR["eps"], AR["r_cut"], 1e-12)
    path = fcb.save_second_order(ifc2, s.n_atoms, 3, str(tmp_path), filename="phi")
    got = fcb.load_force_constants(path)
    assert path.endswith("phi.jld2") and np.array_equal(got["F2"], ifc2)
    assert got["N_atoms"] == s.n_atoms and got["dimension"] == 3 and got["unit"] == ""
    # a non-square (column-major) array keeps its Julia shape
    a = np.asfortranarray(np.arange(24.0).reshape(2, 3, 4, order="F"))
    from fcb200 import hdf5
    p3 = str(tmp_path / "a.jld2")
    hdf5.write(p3, {"a": a, "b": a.astype(np.float32)})
    back = hdf5.read(p3)
    assert back["a"].shape == (2, 3, 4) and np.array_equal(back["a"], a)
    assert back["b"].dtype == np.float32 and np.array_equal(back["b"], a.astype(np.float32))


def _vlen_string_file(path, name, text):
    """A file holding one scalar variable-length UTF-8 string dataset, the
    form JLD2 gives a String: the element (length, global heap collection
    address, object index) points into a "GCOL" collection."""
    import struct
    from fcb200 import hdf5
    payload = text.encode("utf-8")
    gcol_addr, elem_addr = 512, 512 + 4096
    obj = struct.pack("<HHIQ", 1, 1, 0, len(payload)) + payload + b"\x00" * (-len(payload) % 8)
    free = struct.pack("<HHIQ", 0, 0, 0, 4096 - 16 - len(obj) - 16)
    gcol = (b"GCOL" + bytes([1, 0, 0, 0]) + struct.pack("<Q", 4096) + obj + free).ljust(4096, b"\x00")
    base_t = bytes([0x10, 0, 0, 0]) + struct.pack("<I", 1) + struct.pack("<HH", 0, 8)
    vlen_t = bytes([0x19, 0x01, 0x01, 0x00]) + struct.pack("<I", 16) + base_t
    ds = hdf5._object_header([hdf5._message(1, hdf5._dataspace(())), hdf5._message(3, vlen_t, 1),
                              hdf5._message(5, hdf5._fill_value(), 1),
                              hdf5._message(8, hdf5._layout_contiguous(elem_addr, 16))])
    ds_addr = 256
    nm = name.encode()
    root = hdf5._object_header([hdf5._message(2, struct.pack("<BBQQ", 0, 0, hdf5.UNDEF, hdf5.UNDEF)),
                                hdf5._message(10, struct.pack("<BB", 0, 0)),
                                hdf5._message(6, struct.pack("<BBB", 1, 0, len(nm)) + nm + struct.pack("<Q", ds_addr))])
    eof = elem_addr + 16
    sb = hdf5.SIGNATURE + struct.pack("<BBBB", 2, 8, 8, 0) + struct.pack("<QQQQ", 0, hdf5.UNDEF, eof, 48)
    out = bytearray(eof)
    out[0:48] = sb + struct.pack("<I", hdf5.lookup3(sb))
    out[48:48 + len(root)] = root
    out[ds_addr:ds_addr + len(ds)] = ds
    out[gcol_addr:gcol_addr + 4096] = gcol
    out[elem_addr:elem_addr + 16] = struct.pack("<IQI", len(payload), gcol_addr, 1)
    open(path, "wb").write(bytes(out))


def test_reader_takes_variable_length_strings(fcb, tmp_path):
    # the unit string of a file that JLD2 itself wrote is a variable-length
    # string in the global heap
    p = str(tmp_path / "v.jld2")
    _vlen_string_file(p, "unit", "eV Å^-3")
    assert fcb.load_force_constants(p) == {"unit": "eV Å^-3"}

"""Wire formats on either side of the batched path, mirroring ForceConstants.jl
``src/io.jl``.

* ``parse_xyz(path, n_atoms, n_steps)``            io.jl:319-353 — MD trajectory in
* ``save_third_order(psi, n_atoms, D, outpath)``   io.jl:39-68   — IFC3 out
* ``save_second_order(phi, n_atoms, D, outpath)``  io.jl:9-37    — IFC2 out

Text output keeps the reference's header, field order and loop order (1-based
atom and component indices, only non-zero entries); floats are written in
Julia's shortest round-trip form (``1.0e-5``, ``-0.0123``), so a file reads
back bit for bit.  The reference's default format, JLD2, is an HDF5 file with
the keys ``F3``/``F2``, ``N_atoms``, ``dimension`` and ``unit``; ``fmt="JLD2"``
(the default, as in the reference) writes that file through ``fcb200.hdf5``,
and ``load_force_constants`` reads it back.  ``fmt="npz"`` stores the same
keys in a numpy archive.
"""
from __future__ import annotations

import os

import numpy as np

from . import hdf5
from .arrays import is_torch
from .types import DenseForceConstants


def julia_float(x: float) -> str:
    """Julia's `string(::Float64)`: shortest round-trip digits, a `.0` on whole
    mantissas, exponents written as `e-5` / `e16`."""
    s = repr(float(x))
    if s in ("inf", "-inf", "nan"):
        return {"inf": "Inf", "-inf": "-Inf", "nan": "NaN"}[s]
    if "e" in s:
        mant, exp = s.split("e")
        if "." not in mant:
            mant += ".0"
        return f"{mant}e{int(exp)}"
    return s


def _values(ifc):
    v = ifc.values if isinstance(ifc, DenseForceConstants) else ifc
    if is_torch(v):
        v = v.cpu().numpy()
    return np.asarray(v)


def _units(ifc, default: str) -> str:
    return str(ifc.units) if isinstance(ifc, DenseForceConstants) else default


def _round_sig(x: float, digits: int = 7) -> float:
    # round(x, sigdigits = 7)
    return float(f"{x:.{digits - 1}e}") if x != 0.0 else 0.0


_EXT = {"txt": ".txt", "JLD2": ".jld2", "npz": ".npz"}


def _check_out(outpath: str, filename: str, fmt: str) -> str:
    if fmt not in _EXT:
        raise ValueError(f"Invalid format, {fmt}")
    return os.path.join(outpath, filename + _EXT[fmt])


def save_third_order(psi, n_atoms: int, D: int, outpath: str, filename: str = "third_order",
                     fmt: str = "JLD2") -> str:
    """io.jl:39-68.  Returns the path written."""
    v = _values(psi)
    n = n_atoms * D
    assert v.shape == (n, n, n), "Incorrect dimensions"
    path = _check_out(outpath, filename, fmt)
    if fmt == "JLD2":
        hdf5.write(path, {"F3": v, "N_atoms": int(n_atoms), "dimension": int(D), "unit": _units(psi, "")})
        return path
    if fmt == "npz":
        np.savez(path, F3=np.asfortranarray(v), N_atoms=n_atoms, dimension=D, unit=_units(psi, ""))
        return path
    # Ψ[ii,jj,kk], ii = D(i-1)+α (column-major) viewed as axes (α, i, β, j, γ, k);
    # the reference loops i, j, k, α, β, γ (γ fastest).
    six = np.asarray(v).reshape((D, n_atoms, D, n_atoms, D, n_atoms), order="F")
    view = six.transpose(1, 3, 5, 0, 2, 4)
    idx = np.nonzero(view)
    vals = view[idx]
    with open(path, "w") as f:
        f.write(f"#{n_atoms} atoms, Sum Ψ = {julia_float(_round_sig(float(v.sum())))}, "
                f"Units: {_units(psi, '')}\n")
        i, j, k, a, b, c = ((x + 1).tolist() for x in idx)
        vs = [julia_float(x) for x in vals.tolist()]
        f.write("".join(f"{i[t]} {a[t]} {j[t]} {b[t]} {k[t]} {c[t]} {vs[t]}\n" for t in range(len(vs))))
    return path


def save_second_order(phi, n_atoms: int, D: int, outpath: str, filename: str = "second_order",
                      fmt: str = "JLD2") -> str:
    """io.jl:9-37.  Returns the path written."""
    v = _values(phi)
    n = n_atoms * D
    assert v.shape == (n, n), "Incorrect dimensions"
    path = _check_out(outpath, filename, fmt)
    if fmt == "JLD2":
        hdf5.write(path, {"F2": v, "N_atoms": int(n_atoms), "dimension": int(D), "unit": _units(phi, "")})
        return path
    if fmt == "npz":
        np.savez(path, F2=np.asfortranarray(v), N_atoms=n_atoms, dimension=D, unit=_units(phi, ""))
        return path
    four = np.asarray(v).reshape((D, n_atoms, D, n_atoms), order="F")
    view = four.transpose(1, 3, 0, 2)      # loops i, j, α, β
    idx = np.nonzero(view)
    vals = view[idx]
    with open(path, "w") as f:
        f.write(f"#{n_atoms} atoms, Sum Φ = {julia_float(_round_sig(float(v.sum())))}, "
                f"Units: {_units(phi, '')}\n")
        i, j, a, b = ((x + 1).tolist() for x in idx)
        vs = [julia_float(x) for x in vals.tolist()]
        f.write("".join(f"{i[t]} {a[t]} {j[t]} {b[t]} {vs[t]}\n" for t in range(len(vs))))
    return path


def load_third_order_txt(path: str, n_atoms: int, D: int = 3) -> np.ndarray:
    """Reads a file written by save_third_order(fmt="txt") back into a dense
    column-major Ψ (the inverse used by the tests and by callers that keep the
    text format)."""
    n = n_atoms * D
    psi = np.zeros((n, n, n), order="F")
    rows = np.loadtxt(path, comments="#", ndmin=2)
    if rows.size:
        ijk = rows[:, :6].astype(np.int64) - 1
        psi[D * ijk[:, 0] + ijk[:, 1], D * ijk[:, 2] + ijk[:, 3], D * ijk[:, 4] + ijk[:, 5]] = rows[:, 6]
    return psi


def load_force_constants(path: str) -> dict:
    """Reads a file written by save_third_order / save_second_order with
    fmt="JLD2" (or any HDF5 file of plain datasets in its root group):
    name -> value, arrays in Julia's column-major shape."""
    return hdf5.read(path)


def parse_xyz(path: str, n_atoms: int, n_steps: int):
    """io.jl:319-353: frames of two header lines followed by n_atoms lines
    `id x y z`.  Returns (positions, ids): positions[s] is a (k, 3) float64
    array (every column after the id, as the reference's `posn...`) and ids[s]
    the atom ids of frame s, for s < n_steps.  The reference's state machine
    is kept: blank lines are skipped (readdlm), a frame the file does not hold
    comes back empty and a truncated last frame with the atoms it has, and an
    atom line past frame n_steps raises IndexError (Julia's BoundsError), as
    does an id that is not an integer raise ValueError (InexactError)."""
    rows = [[] for _ in range(n_steps)]
    ids = [[] for _ in range(n_steps)]
    header_size = 2
    line_num = 0
    step = 0
    with open(path) as f:
        for raw in f:
            tok = raw.split()
            if not tok:
                continue
            if line_num in (0, 1):
                line_num += 1
                continue
            if step >= n_steps:
                raise IndexError(f"attempt to access {n_steps}-element Vector at index [{step + 1}]")
            idv = float(tok[0])
            if not idv.is_integer():
                raise ValueError(f"InexactError: Int64({tok[0]})")
            ids[step].append(int(idv))
            rows[step].append([float(x) for x in tok[1:]])
            line_num += 1
            if line_num == n_atoms + header_size:
                line_num = 0
                step += 1
    positions = [np.array(r, dtype=np.float64).reshape(len(r), -1) if r else np.empty((0, 3)) for r in rows]
    return positions, [np.array(i, dtype=np.int64) for i in ids]

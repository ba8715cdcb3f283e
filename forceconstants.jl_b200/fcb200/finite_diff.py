"""Finite-difference force constants mirroring ForceConstants.jl
``src/finitediff/``, computed on the GPU (``fcb200_fd_*``).

* ``third_order_finite_diff_eng(sys, pot, atom_idxs, cartesian_idxs, h)``
  third_order_FD.jl:43-113 — one element, 1-based indices as the reference
* ``third_order_fd(sys, pot, elems, h)`` — many elements at once, 0-based rows
  (i, α, j, β, k, γ); NaN where the reference has no stencil
* ``second_order(sys, pot, FiniteDiffCalculator(tol, r_cut))`` goes through
  ``ifc.second_order`` (second_order_FD.jl:3-79)
"""
from __future__ import annotations

import warnings

import numpy as np

from . import _lib
from .arrays import ptr
from .types import FD_STEP, LJ, StillingerWeberSilicon


def third_order_fd(sys, pot, elems, h: float = FD_STEP, device: int = 0) -> np.ndarray:
    e = np.ascontiguousarray(elems, dtype=np.int64).reshape(-1, 6)
    out = np.empty(e.shape[0])
    L = _lib.lib()
    if isinstance(pot, LJ):
        st = L.fcb200_fd_third_order_lj(_lib.handle(device), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes),
                                        float(pot.sigma), float(pot.eps), float(pot.r_cut), ptr(e), e.shape[0],
                                        float(h), ptr(out), 0)
    elif isinstance(pot, StillingerWeberSilicon):
        st = L.fcb200_fd_third_order_sw(_lib.handle(device), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes),
                                        ptr(e), e.shape[0], float(h), ptr(out), 0)
    else:
        raise TypeError(f"no finite-difference energy for {type(pot).__name__}")
    if st == _lib.FCB_ERR_ARG:
        raise AssertionError(_lib.last_error()[1])
    _lib.check(st)
    return out


def third_order_finite_diff_eng(sys, pot, atom_idxs, cartesian_idxs, h: float = FD_STEP):
    """third_order_FD.jl:43-113 (1-based atom and Cartesian indices).  Returns
    None, with a warning, for the arrangements the reference does not
    implement (i == j != k, j == k != i)."""
    assert len(atom_idxs) == 3
    assert len(cartesian_idxs) == 3
    N = sys.n_atoms
    assert all(1 <= a <= N for a in atom_idxs), f"Atom indexes out of range, must be in 1:{N}"
    assert all(1 <= c <= 3 for c in cartesian_idxs), "Cartesian indices must be 1, 2, or 3"
    row = [v - 1 for pair in zip(atom_idxs, cartesian_idxs) for v in pair]
    v = float(third_order_fd(sys, pot, [row], h)[0])
    if np.isnan(v):
        warnings.warn("Not implemented")
        return None
    return v


def second_order_fd_(ifc2, sys, pot, calc, device: int = 0):
    """second_order! with the FiniteDiffCalculator (then apply_tols!, as
    second_order does)."""
    L = _lib.lib()
    if isinstance(pot, LJ):
        _lib.check(L.fcb200_fd_second_order_lj(_lib.handle(device), ptr(sys.positions), sys.n_atoms,
                                               ptr(sys.box_sizes), float(pot.sigma), float(pot.eps),
                                               float(pot.r_cut), float(calc.r_cut), float(calc.tol), float(calc.h),
                                               ptr(ifc2), 0))
    elif isinstance(pot, StillingerWeberSilicon):
        _lib.check(L.fcb200_fd_second_order_sw(_lib.handle(device), ptr(sys.positions), sys.n_atoms,
                                               ptr(sys.box_sizes), float(calc.r_cut), float(calc.tol),
                                               float(calc.h), ptr(ifc2), 0))
    else:
        raise TypeError(f"no finite-difference energy for {type(pot).__name__}")
    return ifc2

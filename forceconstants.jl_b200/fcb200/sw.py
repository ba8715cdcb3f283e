"""Stillinger-Weber silicon through the C ABI (the reference's AutoDiffCalculator
path: src/autodiff/third_order_AD.jl:71-224, second_order_AD.jl:40-110)."""
from __future__ import annotations

import numpy as np

from . import _lib
from .arrays import device_index, ptr, stream_ptr

COS0_GENERATED = -0.333333333333   # cosθ₀ as written in the reference's generated kernels
COS0_IIK = -1.0 / 3.0              # cosθ₀ of the run-time iik block (the potential's own value)


def _cos0(pot):
    return np.array([COS0_GENERATED, float(pot.cos0)], dtype=np.float64)


def third_order_sw_(psi, sys, pot, calc, masses=None, mass_weighted=False, psi32_mw=None):
    n = 3 * sys.n_atoms
    if tuple(psi.shape) != (n, n, n):
        raise AssertionError("size(Ψ) == (D*N_atoms, D*N_atoms, D*N_atoms)")
    if not calc.r_cut <= pot.r_cut:
        raise AssertionError("For AutoDiff SW silicon force constant cutoff must be less than potential cutoff")
    m = sys.masses if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
    need_m = mass_weighted or psi32_mw is not None
    c0 = _cos0(pot)
    _lib.check(_lib.lib().fcb200_third_order_sw(
        _lib.handle(device_index(psi)), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(calc.r_cut),
        float(calc.tol), ptr(c0), ptr(m) if need_m else 0, ptr(psi), ptr(psi32_mw),
        _lib.FCB_PSI_MASS_WEIGHTED if mass_weighted else 0, stream_ptr(psi)))
    return psi


def second_order_sw_(ifc2, sys, pot, calc, masses=None):
    if not calc.r_cut <= pot.r_cut:
        raise AssertionError("For AutoDiff SW silicon force constant cutoff must be less than potential cutoff")
    m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
    c0 = _cos0(pot)
    _lib.check(_lib.lib().fcb200_second_order_sw(
        _lib.handle(device_index(ifc2)), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(calc.r_cut),
        float(calc.tol), ptr(c0), ptr(m), ptr(ifc2), stream_ptr(ifc2)))
    return ifc2

"""Gradient of a scalar of K3 with respect to positions and LJ σ, ε (φ frozen).

The Python counterpart of the ChainRulesCore `rrule` a Julia host would wrap
around ``fcb200_mcc3_adjoint_lj``: given the cotangent W of K3 (over the first
``n_modes`` modes on every axis), returns ∂L/∂positions, ∂L/∂σ, ∂L/∂ε for
L = Σ W·K3, together with L.  ``precision`` is the arithmetic of
G = W ×₁φᵀ ×₂φᵀ ×₃φᵀ: "fp32", "tf32x3", "bf16x3" (as for mcc3) or "fp64".
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .arrays import as_julia, device_index, is_torch, ptr, stream_ptr


def mcc3_adjoint_lj(sys, pot, calc, phi, W, precision: str = "fp64"):
    M = int(W.shape[0])
    W = as_julia(W, np.float32)
    phi = as_julia(phi, np.float32)
    dpos = np.zeros(3 * sys.n_atoms)
    dsig, deps, L = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    dev = device_index(W) if is_torch(W) else device_index(phi)
    _lib.check(_lib.lib().fcb200_mcc3_adjoint_lj(
        _lib.handle(dev), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(pot.sigma), float(pot.eps),
        float(calc.r_cut), ptr(sys.masses), ptr(phi), M, ptr(W), _lib.ADJOINT_PRECISIONS[precision], ptr(dpos),
        ctypes.byref(dsig), ctypes.byref(deps), ctypes.byref(L), stream_ptr(W) or stream_ptr(phi)))
    return {"dpos": dpos.reshape(-1, 3), "dsigma": dsig.value, "deps": deps.value, "L": L.value}

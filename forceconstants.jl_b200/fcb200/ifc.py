"""Force-constant front end mirroring ForceConstants.jl ``src/ifc.jl``.

Names and argument meaning follow the reference; Julia's mutating ``f!`` is
spelled ``f_`` here.  Every function computes through ``libfcb200.so`` on the
GPU; there is no CPU path.

* ``third_order(sys, pot, calc)``            ifc.jl:20-35
* ``third_order_(psi, sys, pot, calc)``      third_order!  (analytical: third_order_analytical.jl:4-69,
                                             SW AD: autodiff/third_order_AD.jl:71-170)
* ``mass_weight_third_order_(ifc3, masses)`` third_order_analytical.jl:185-214
* ``second_order(sys, pot, calc)``           ifc.jl:3-18
* ``dynamical_matrix(sys, pot, calc)``       dynmat.jl:5-33
* ``get_modes(dynmat, n_rigid=3)``           dynmat.jl:123-141 (cuSOLVER syevd on the GPU)
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .arrays import as_julia, device_index, device_of, is_torch, julia_empty, ptr, stream_ptr
from .types import (LJ, AnalyticalCalculator, AutoDiffCalculator, DenseForceConstants, StillingerWeberSilicon,
                    SuperCellSystem)


def _check_cut(sys: SuperCellSystem, r_cut: float) -> None:
    # third_order_analytical.jl:7 — the reference asserts r_cut < L (not L/2).
    if not np.all(r_cut < sys.box_sizes):
        raise AssertionError("Cutoff larger than L/2")


def third_order_(psi, sys: SuperCellSystem, pot, calc, n_threads: int | None = None, masses=None,
                 mass_weighted: bool = False, psi32_mw=None):
    """Fill ``psi`` (n×n×n, column-major; numpy or CUDA torch) with Ψ after ASR
    and the tolerance cutoff.  ``n_threads`` is accepted and ignored.

    Extensions beyond the reference (all optional): ``mass_weighted`` writes
    Ψ/sqrt(m_i m_j m_k) instead; ``psi32_mw`` receives the FP32 mass-weighted
    copy that ``mcc3`` consumes, from the same pass.
    """
    del n_threads
    if isinstance(pot, StillingerWeberSilicon):
        from .sw import third_order_sw_
        return third_order_sw_(psi, sys, pot, calc, masses=masses, mass_weighted=mass_weighted,
                               psi32_mw=psi32_mw)
    if not isinstance(pot, LJ):
        raise TypeError(f"no third_order! method for {type(pot).__name__}")
    if not isinstance(calc, (AnalyticalCalculator, AutoDiffCalculator)):
        raise TypeError(f"no third_order! method for {type(calc).__name__}")
    n = 3 * sys.n_atoms
    if tuple(psi.shape) != (n, n, n):
        raise AssertionError("size(Ψ) == (D*N_atoms, D*N_atoms, D*N_atoms)")
    if isinstance(calc, AnalyticalCalculator):
        _check_cut(sys, pot.r_cut)      # the reference asserts on the potential's cutoff
    _check_cut(sys, calc.r_cut)         # the pair loop's single minimum image needs r_cut < L
    m = sys.masses if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
    need_m = mass_weighted or psi32_mw is not None
    flags = _lib.FCB_PSI_MASS_WEIGHTED if mass_weighted else 0
    dev = device_index(psi)
    _lib.check(_lib.lib().fcb200_third_order_lj(
        _lib.handle(dev), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(pot.sigma), float(pot.eps),
        float(calc.r_cut), float(calc.tol), ptr(m) if need_m else 0, ptr(psi), ptr(psi32_mw), flags,
        stream_ptr(psi)))
    return psi


def third_order(sys: SuperCellSystem, pot, calc, n_threads: int | None = None, check_asr: bool = False,
                device: str = "cpu") -> DenseForceConstants:
    """ifc.jl:20-35.  ``device="cpu"`` returns a host array like the reference;
    ``device="cuda"`` keeps Ψ on the GPU as a torch tensor."""
    n = 3 * sys.n_atoms
    psi = julia_empty((n, n, n), np.float64, device)
    third_order_(psi, sys, pot, calc, n_threads=n_threads)
    if check_asr:
        vals = psi if not is_torch(psi) else psi.cpu().numpy()
        assert asr_satisfied(vals, sys.n_atoms, 3, calc.tol), \
            "ASR not satisfied for third order force constants, please report this"
    return DenseForceConstants(psi, f"{pot.energy_unit} {pot.length_unit}^-3", calc.tol)


def mass_weight_third_order_(ifc3: DenseForceConstants, masses) -> DenseForceConstants:
    """third_order_analytical.jl:185-214: Ψ[ii,jj,kk] /= sqrt(m_i m_j m_k) for
    non-zero entries, in place; the unit is divided by the mass unit once (the
    reference's own convention)."""
    m = np.ascontiguousarray(np.asarray(masses, dtype=np.float64).reshape(-1))
    n = ifc3.values.shape[0]
    if n % m.shape[0] != 0 or n // m.shape[0] not in (1, 2, 3):
        raise AssertionError("D ∈ [1,2,3]")
    if n // m.shape[0] != 3:
        raise NotImplementedError("only D = 3 is supported")
    psi = ifc3.values
    dev = device_index(psi)
    _lib.check(_lib.lib().fcb200_mass_weight3(_lib.handle(dev), ptr(psi), ptr(m), m.shape[0], stream_ptr(psi)))
    ifc3.units = f"{ifc3.units} u^-1"
    return ifc3


def second_order_(ifc2, sys: SuperCellSystem, pot, calc, n_threads: int | None = None, masses=None):
    del n_threads
    from .types import FiniteDiffCalculator
    if isinstance(calc, FiniteDiffCalculator):
        if masses is not None:
            raise NotImplementedError("mass weighting of finite-difference IFC2: divide by sqrt(m_i m_j) after")
        from .finite_diff import second_order_fd_
        return second_order_fd_(ifc2, sys, pot, calc, device=device_index(ifc2))
    if isinstance(pot, StillingerWeberSilicon):
        from .sw import second_order_sw_
        return second_order_sw_(ifc2, sys, pot, calc, masses=masses)
    if not isinstance(pot, LJ):
        raise TypeError(f"no second_order! method for {type(pot).__name__}")
    if isinstance(calc, AutoDiffCalculator) and not calc.r_cut <= pot.r_cut:
        # second_order_AD.jl:4
        raise AssertionError("Calculator r_cut must be less than potential r_cut")
    dev = device_index(ifc2)
    m = None if masses is None else np.ascontiguousarray(masses, dtype=np.float64)
    _lib.check(_lib.lib().fcb200_second_order_lj(
        _lib.handle(dev), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(pot.sigma), float(pot.eps),
        float(calc.r_cut), float(calc.tol), ptr(m), ptr(ifc2), stream_ptr(ifc2)))
    return ifc2


def second_order(sys: SuperCellSystem, pot, calc, n_threads: int | None = None, check_asr: bool = False,
                 check_symmetry: bool = False, device: str = "cpu") -> DenseForceConstants:
    """ifc.jl:3-18."""
    n = 3 * sys.n_atoms
    ifc2 = julia_empty((n, n), np.float64, device)
    second_order_(ifc2, sys, pot, calc, n_threads=n_threads)
    vals = ifc2 if not is_torch(ifc2) else ifc2.cpu().numpy()
    if check_asr:
        assert asr_satisfied(vals, sys.n_atoms, 3, calc.tol), \
            "ASR not satisfied for second order force constants, please report this"
    if check_symmetry:
        assert np.array_equal(vals, vals.T), "IFC were not symmetric, please report this"
    return DenseForceConstants(ifc2, f"{pot.energy_unit} {pot.length_unit}^-2", calc.tol)


def dynamical_matrix(sys: SuperCellSystem, pot, calc, device: str = "cpu") -> DenseForceConstants:
    """dynmat.jl:5-33: second order divided by sqrt(m_i m_j) (tolerance 0)."""
    n = 3 * sys.n_atoms
    dyn = julia_empty((n, n), np.float64, device)
    second_order_(dyn, sys, pot, calc, masses=sys.masses)
    return DenseForceConstants(dyn, f"{pot.energy_unit} {pot.length_unit}^-2 u^-1", 0.0)


def get_modes(dynmat, num_rigid_translation: int = 3, phi32: bool = False):
    """dynmat.jl:123-141: ascending eigenvalues and orthonormal eigenvectors of
    the Hermitian dynamical matrix; the ``num_rigid_translation`` eigenvalues
    nearest zero (stable order of |λ|) are set to 0.  Solved on the GPU
    (``fcb200_get_modes``, cuSOLVER syevd).  Outputs live where the input
    lives (numpy in, numpy out; CUDA tensor in, CUDA tensors out).  With
    ``phi32=True`` the FP32 copy of the eigenvectors — the φ operand of
    ``mcc3`` — is returned as a third value."""
    vals = dynmat.values if isinstance(dynmat, DenseForceConstants) else dynmat
    vals = as_julia(vals, np.float64)
    if vals.ndim != 2 or vals.shape[0] != vals.shape[1]:
        raise ValueError("dynmat must be square")
    n = int(vals.shape[0])
    dev = device_of(vals)
    w = julia_empty((n,), np.float64, dev)
    v = julia_empty((n, n), np.float64, dev)
    f = julia_empty((n, n), np.float32, dev) if phi32 else None
    _lib.check(_lib.lib().fcb200_get_modes(
        _lib.handle(device_index(vals)), ptr(vals), n, int(num_rigid_translation), ptr(w), ptr(v), ptr(f),
        stream_ptr(vals)))
    return (w, v, f) if phi32 else (w, v)


def asr_satisfied(ifc, n_atoms: int, D: int, tol: float, verbose: bool = False) -> bool:
    """asr.jl:43-74 (host check).  Like the reference, a slice fails when its
    sum exceeds ``tol`` (no absolute value)."""
    a = np.asarray(ifc)
    if a.ndim == 2:
        for i in range(n_atoms):
            for al in range(D):
                for be in range(D):
                    s = a[D * i + al, be::D].sum()
                    if s > tol:
                        if verbose:
                            print(f"Set i = {i + 1}, α = {al + 1}, β = {be + 1} does not satisfy ASR. Sum was: {s}")
                        return False
        return True
    ok = True
    for k in range(a.shape[2]):
        ok &= asr_satisfied(a[:, :, k], n_atoms, D, tol, verbose)
    return ok


__all__ = ["third_order", "third_order_", "mass_weight_third_order_", "second_order", "second_order_",
           "dynamical_matrix", "get_modes", "asr_satisfied", "as_julia", "device_of"]

"""ORACLE — test infrastructure only.  Python driver for the CPU restatement.

Wraps ``oracle/liboracle.so`` (built from ``lj_oracle.c`` / ``sw_oracle.c`` by
``oracle/build.py``) and adds the pieces of the reference path that are plain
dense linear algebra, restated with numpy in FP64:

* ``dynamical_matrix`` / ``get_modes``   — src/dynmat.jl:5-33, 123-131
* ``mcc3``                                — src/mcc.jl:29-51 (three mode products)
* ``mcc3_blocked``                        — src/mcc.jl:89-134 (block semantics)

All tensors use Julia's index semantics: ``psi[i, j, k]`` is the reference's
``Ψ[i,j,k]`` (0-based here).  Arrays returned from C are Fortran-ordered views so
that their memory layout is the reference's column-major layout.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_D = ctypes.c_double
_I64 = ctypes.c_int64
_PD = ctypes.POINTER(ctypes.c_double)
_PF = ctypes.POINTER(ctypes.c_float)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            import sys
            sys.path.insert(0, HERE)
            from build import build_oracle
            build_oracle()
        L = ctypes.CDLL(path)
        L.oracle_third_order_lj.argtypes = [_PD, _I64, _PD, _D, _D, _D, _D, _PD]
        L.oracle_third_order_lj.restype = ctypes.c_int
        L.oracle_third_order_lj_pairs.argtypes = [_PD, _I64, _PD, _D, _D, _D, _PD]
        L.oracle_second_order_lj_full.argtypes = [_PD, _I64, _PD, _D, _D, _D, _D, _PD]
        L.oracle_second_order_lj_full.restype = ctypes.c_int
        L.oracle_mass_weight3.argtypes = [_PD, _PD, _I64]
        L.oracle_apply_tols.argtypes = [_PD, _I64, _D]
        L.oracle_asr3.argtypes = [_PD, _I64]
        L.oracle_cast_f32.argtypes = [_PD, _PF, _I64]
        L.oracle_lj_derivs.argtypes = [_D, _D, _D, _PD]
        L.oracle_set_num_threads.argtypes = [ctypes.c_int]
        L.oracle_num_threads.restype = ctypes.c_int
        _sw_signatures(L)
        _lib = L
    return _lib


def _sw_signatures(L):
    L.oracle_third_order_sw.argtypes = [_PD, _I64, _PD, _PD, _D, _D, _PD]
    L.oracle_third_order_sw.restype = ctypes.c_int
    L.oracle_second_order_sw.argtypes = [_PD, _I64, _PD, _PD, _D, _D, _PD]
    L.oracle_second_order_sw.restype = ctypes.c_int
    L.oracle_sw_triplet_blocks.argtypes = [_PD, _PD, _PD]
    L.oracle_sw_triplet_blocks2.argtypes = [_PD, _PD, _PD]
    L.oracle_sw_pair_block3.argtypes = [_PD, _PD]
    L.oracle_sw_pair_block2.argtypes = [_PD, _PD]
    L.oracle_sw_rcut.restype = ctypes.c_double


_ref = None


def ref_lib():
    """oracle/_ref/libswref.so: the same SW loop driven by the reference's own
    generated derivative kernels (built only where the reference checkout is
    present; None otherwise)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libswref.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        _sw_signatures(L)
        _ref = L
    return _ref


COS0_GEN = -0.333333333333
COS0_IIK = -1.0 / 3.0


def sw_blocks(r9, cos0=(COS0_GEN, COS0_IIK), use_ref=False):
    """The 7 third-derivative blocks (iij, ijj, iik, ikk, jjk, jkk, ijk) of one
    SW triplet from 9 absolute coordinates; column-major 3×3×3 each."""
    L = ref_lib() if use_ref else lib()
    r9 = np.ascontiguousarray(r9, dtype=np.float64)
    c = np.ascontiguousarray(cos0, dtype=np.float64)
    out = np.zeros(7 * 27)
    L.oracle_sw_triplet_blocks(_pd(r9), _pd(c), _pd(out))
    return out.reshape(7, 27)


def sw_pair_block(r3, use_ref=False):
    L = ref_lib() if use_ref else lib()
    r3 = np.ascontiguousarray(r3, dtype=np.float64)
    out = np.zeros(27)
    L.oracle_sw_pair_block3(_pd(r3), _pd(out))
    return out


def _pd(a):
    return a.ctypes.data_as(_PD)


def set_threads(t: int) -> None:
    lib().oracle_set_num_threads(int(t))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def _pos(pos):
    pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(-1, 3))
    return pos, pos.shape[0]


def third_order_lj(pos, box, sigma, eps, r_cut, tol):
    """ifc.jl:20-35 with the analytical LJ calculator: unweighted Ψ (n×n×n)."""
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n = 3 * N
    psi = np.empty(n * n * n, dtype=np.float64)
    rc = lib().oracle_third_order_lj(_pd(pos), N, _pd(box), sigma, eps, r_cut, tol, _pd(psi))
    if rc != 0:
        raise ValueError("Cutoff larger than L/2")
    return psi.reshape((n, n, n), order="F")


def second_order_lj(pos, box, sigma, eps, r_cut, tol):
    """ifc.jl:3-18 with the analytical LJ calculator: IFC2 (n×n)."""
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n = 3 * N
    ifc2 = np.empty(n * n, dtype=np.float64)
    lib().oracle_second_order_lj_full(_pd(pos), N, _pd(box), sigma, eps, r_cut, tol, _pd(ifc2))
    return ifc2.reshape((n, n), order="F")


def mass_weight_third_order(psi, masses):
    """third_order_analytical.jl:185-214, in place on a Fortran-ordered array."""
    assert psi.flags.f_contiguous and psi.dtype == np.float64
    masses = np.ascontiguousarray(masses, dtype=np.float64)
    flat = psi.reshape(-1, order="F")
    lib().oracle_mass_weight3(_pd(flat), _pd(masses), masses.shape[0])
    return psi


def third_order_sw(pos, box, r_cut, tol, cos0_generated=-0.333333333333, cos0_iik=-1.0 / 3.0, use_ref=False):
    """third_order_AD.jl:71-170 + ifc.jl:20-35 for Stillinger-Weber silicon."""
    L = ref_lib() if use_ref else lib()
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n = 3 * N
    psi = np.empty(n * n * n, dtype=np.float64)
    cos0 = np.array([cos0_generated, cos0_iik], dtype=np.float64)
    rc = L.oracle_third_order_sw(_pd(pos), N, _pd(box), _pd(cos0), r_cut, tol, _pd(psi))
    if rc != 0:
        raise ValueError("force-constant cutoff must be below the SW cutoff and the box")
    return psi.reshape((n, n, n), order="F")


def second_order_sw(pos, box, r_cut, tol, cos0_generated=-0.333333333333, use_ref=False):
    """second_order_AD.jl:40-110 + ifc.jl:3-18 for Stillinger-Weber silicon."""
    L = ref_lib() if use_ref else lib()
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n = 3 * N
    ifc2 = np.empty(n * n, dtype=np.float64)
    cos0 = np.array([cos0_generated, cos0_generated], dtype=np.float64)
    rc = L.oracle_second_order_sw(_pd(pos), N, _pd(box), _pd(cos0), r_cut, tol, _pd(ifc2))
    if rc != 0:
        raise ValueError("force-constant cutoff must be below the SW cutoff and the box")
    return ifc2.reshape((n, n), order="F")


def dynamical_matrix(ifc2, masses):
    """dynmat.jl:5-33: divide by sqrt(m_i m_j) per 3×3 block."""
    m = np.repeat(np.asarray(masses, dtype=np.float64), 3)
    return ifc2 / np.sqrt(np.outer(m, m))


def get_modes(dynmat, num_rigid_translation=3):
    """dynmat.jl:123-131: ascending eigen-decomposition, rigid modes zeroed."""
    w, v = np.linalg.eigh(dynmat)
    idx = np.argsort(np.abs(w), kind="stable")
    w = w.copy()
    w[idx[:num_rigid_translation]] = 0.0
    return w, v


def mcc3(psi, phi, modes=None):
    """mcc.jl:29-51 in FP64: K1[n,j,k], K2[n,k,m], K3[n,m,l].

    ``modes`` = (lo, hi) restricts every mode axis to phi[:, lo:hi].
    """
    psi = np.asarray(psi, dtype=np.float64)
    phi = np.asarray(phi, dtype=np.float64)
    if modes is not None:
        phi = phi[:, modes[0]:modes[1]]
    k1 = np.tensordot(phi, psi, axes=([0], [0]))      # [n, j, k]
    k2 = np.tensordot(k1, phi, axes=([1], [0]))       # [n, k, m]
    k3 = np.tensordot(k2, phi, axes=([1], [0]))       # [n, m, l]
    return k3


def mcc3_blocked(psi, phi, block_size):
    """mcc.jl:89-134: assemble K3 from (n/b)³ blocks with column-sliced phi."""
    n = phi.shape[0]
    if n % block_size != 0 or block_size <= 0:
        raise ValueError("size(phi,1) must be a multiple of block_size")
    nb = n // block_size
    out = np.zeros((n, n, n), dtype=np.float64)
    for a in range(nb):
        ra = slice(a * block_size, (a + 1) * block_size)
        k1 = np.tensordot(phi[:, ra], psi, axes=([0], [0]))
        for b in range(nb):
            rb = slice(b * block_size, (b + 1) * block_size)
            k2 = np.tensordot(k1, phi[:, rb], axes=([1], [0]))
            for c in range(nb):
                rc = slice(c * block_size, (c + 1) * block_size)
                out[ra, rb, rc] = np.tensordot(k2, phi[:, rc], axes=([1], [0]))
    return out


def lj_derivs(sigma, eps, r):
    d = np.zeros(4)
    lib().oracle_lj_derivs(sigma, eps, r, _pd(d))
    return d

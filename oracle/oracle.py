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
        L.oracle_third_order_lj_slab.argtypes = [_PD, _I64, _PD, _D, _D, _D, _D, _I64, _I64, _PD]
        L.oracle_third_order_lj_slab.restype = ctypes.c_int
        L.oracle_second_order_lj_full.argtypes = [_PD, _I64, _PD, _D, _D, _D, _D, _PD]
        L.oracle_second_order_lj_full.restype = ctypes.c_int
        L.oracle_mass_weight3.argtypes = [_PD, _PD, _I64]
        L.oracle_apply_tols.argtypes = [_PD, _I64, _D]
        L.oracle_asr3.argtypes = [_PD, _I64]
        L.oracle_cast_f32.argtypes = [_PD, _PF, _I64]
        L.oracle_lj_derivs.argtypes = [_D, _D, _D, _PD]
        L.oracle_set_num_threads.argtypes = [ctypes.c_int]
        L.oracle_nearest_mirror.argtypes = [_PD, _PD]
        L.oracle_num_threads.restype = ctypes.c_int
        _sw_signatures(L)
        _fd_signatures(L)
        _lib = L
    return _lib


def _fd_signatures(L):
    _P64 = ctypes.POINTER(ctypes.c_int64)
    L.oracle_fd_third_order.argtypes = [ctypes.c_int, _PD, _I64, _PD, _D, _D, _D, _P64, _I64, _D, _PD]
    L.oracle_fd_second_order.argtypes = [ctypes.c_int, _PD, _I64, _PD, _D, _D, _D, _D, _D, _PD]
    L.oracle_fd_energy.argtypes = [ctypes.c_int, _PD, _I64, _PD, _D, _D, _D]
    L.oracle_fd_energy.restype = _D


FD_STEP = 0.04 * 0.5291772109   # the reference's default h: 0.04 bohr in Å (third_order_FD.jl:43)


def fd_third_order(kind, pos, box, elems, h=FD_STEP, sigma=0.0, eps=0.0, r_cut=0.0):
    """third_order_finite_diff_eng (src/finitediff/third_order_FD.jl:43-113) for the
    elements (i, α, j, β, k, γ) (0-based rows of `elems`); kind "lj" or "sw".
    Total-energy stencils as the reference; NaN where it has none."""
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    e = np.ascontiguousarray(elems, dtype=np.int64).reshape(-1, 6)
    out = np.empty(e.shape[0])
    lib().oracle_fd_third_order(0 if kind == "lj" else 1, _pd(pos), N, _pd(box), sigma, eps, r_cut,
                                e.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), e.shape[0], h, _pd(out))
    return out


def fd_second_order(kind, pos, box, calc_rcut, h=FD_STEP, sigma=0.0, eps=0.0, r_cut=0.0):
    """second_order! with the FiniteDiffCalculator (src/finitediff/second_order_FD.jl:3-79,
    ASR src/asr.jl:3-17): n×n column-major."""
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n = 3 * N
    out = np.empty(n * n)
    lib().oracle_fd_second_order(0 if kind == "lj" else 1, _pd(pos), N, _pd(box), sigma, eps, r_cut, calc_rcut,
                                 h, _pd(out))
    return out.reshape((n, n), order="F")


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


def third_order_lj_slab(pos, box, sigma, eps, r_cut, tol, j0, j1):
    """The columns jj in [j0, j1) of the middle index of third_order_lj
    (ifc.jl:20-35): an n × (j1 - j0) × n Fortran array equal, entry for entry,
    to ``third_order_lj(...)[:, j0:j1, :]`` (lj_oracle.c, oracle_third_order_lj_slab)."""
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n, w = 3 * N, int(j1) - int(j0)
    out = np.empty(n * w * n, dtype=np.float64)
    rc = lib().oracle_third_order_lj_slab(_pd(pos), N, _pd(box), sigma, eps, r_cut, tol, int(j0), int(j1), _pd(out))
    if rc == -1:
        raise ValueError("Cutoff larger than L/2")
    if rc != 0:
        raise ValueError("slab outside [0, n)")
    return out.reshape((n, w, n), order="F")


def lj_slabs(pos, box, sigma, eps, r_cut, tol, atoms_per_slab=8):
    """Yields (j0, j1, slab) over the whole middle index, slab by slab."""
    N = np.asarray(pos).reshape(-1, 3).shape[0]
    n = 3 * N
    for a0 in range(0, N, atoms_per_slab):
        j0, j1 = 3 * a0, min(n, 3 * (a0 + atoms_per_slab))
        yield j0, j1, third_order_lj_slab(pos, box, sigma, eps, r_cut, tol, j0, j1)


def mass_weight_slab(slab, masses, j0, f32=False):
    """third_order_analytical.jl:185-214 on an n × w × n slab (columns j0..):
    non-zero entries divided by sqrt((m_i·m_j)·m_k), the oracle's expression;
    with ``f32`` the weighted values are rounded to FP32 (held in FP64)."""
    m = np.repeat(np.asarray(masses, dtype=np.float64), 3)
    n, w = slab.shape[0], slab.shape[1]
    flat = slab.reshape(-1, order="F")
    idx = np.flatnonzero(flat)
    i, rest = idx % n, idx // n
    j, k = rest % w, rest // w
    vals = flat[idx] / np.sqrt((m[i] * m[j0 + j]) * m[k])
    if f32:
        vals = vals.astype(np.float32).astype(np.float64)
    out = np.zeros(flat.shape[0])
    out[idx] = vals
    return out.reshape(slab.shape, order="F")


def mcc3_windows_lj(pos, box, sigma, eps, r_cut, tol, masses, phi, windows, atoms_per_slab=8, f32=True,
                    on_slab=None):
    """K3 over mode windows, K3[p, q, s] = Σ_ijk Ψ_mw[i,j,k] φ[i,p] φ[j,q] φ[k,s]
    for p ∈ P, q ∈ Q, s ∈ S (mcc.jl:29-51 in FP64), accumulated over slabs of
    the middle index so that the dense Ψ of a large cell is never held whole.
    Ψ_mw is rounded to FP32 first when ``f32`` (the reference's
    CuArray{Float32} operand, README.md:73-75).  ``windows`` is a list of
    (P, Q, S) index arrays; ``on_slab(j0, j1, slab)`` sees every unweighted slab."""
    phi = np.asarray(phi, dtype=np.float64)
    outs = [np.zeros((len(P), len(Q), len(S))) for P, Q, S in windows]
    for j0, j1, slab in lj_slabs(pos, box, sigma, eps, r_cut, tol, atoms_per_slab):
        if on_slab is not None:
            on_slab(j0, j1, slab)
        mw = mass_weight_slab(slab, masses, j0, f32=f32)
        n, w = mw.shape[0], mw.shape[1]
        m2 = mw.reshape(n, w * n, order="F")                          # [i, (jl, k)], a view
        for (P, Q, S), out in zip(windows, outs):
            t = np.ascontiguousarray(phi[:, P].T) @ m2                # [p, jl + w·k]
            t = np.matmul(t.reshape(len(P), n, w).transpose(0, 2, 1), phi[:, S])   # [p, jl, s]
            out += np.einsum("pjs,jq->pqs", t, phi[j0:j1][:, Q], optimize=True)
    return outs


def second_order_lj(pos, box, sigma, eps, r_cut, tol):
    """ifc.jl:3-18 with the analytical LJ calculator: IFC2 (n×n)."""
    pos, N = _pos(pos)
    box = np.ascontiguousarray(box, dtype=np.float64)
    n = 3 * N
    ifc2 = np.empty(n * n, dtype=np.float64)
    lib().oracle_second_order_lj_full(_pd(pos), N, _pd(box), sigma, eps, r_cut, tol, _pd(ifc2))
    return ifc2.reshape((n, n), order="F")


def _ref_lj_kernel(name):
    L = ref_lib()
    if L is None:
        return None
    f = getattr(L, name)
    f.restype = None
    f.argtypes = [_PD, _PD]
    return f


def _lj_pairs_ad(pos, box, r_cut):
    """Pairs i < j within r_cut at the single minimum image, in the order of
    the reference's loop (i ascending, then j), with r_ij = r_i - r_j mirrored
    by nearest_mirror! (helper_funcs.jl:7-17)."""
    pos, N = _pos(pos)
    box = np.asarray(box, dtype=np.float64)
    out = []
    for i in range(N):
        r = pos[i] - pos[i + 1:]
        r = np.where(r > box / 2, r - box, np.where(r < -box / 2, r + box, r))
        d2 = np.sum(r * r, axis=1)
        for j in np.nonzero(d2 < r_cut * r_cut)[0]:
            out.append((i, i + 1 + int(j), np.ascontiguousarray(r[j])))
    return out, N


def second_order_lj_ad_ref(pos, box, r_cut, tol):
    """second_order! with the AutoDiffCalculator for LJ
    (src/autodiff/second_order_AD.jl:1-37) driven by the reference's own
    generated Hessian kernel (H2_exec_LJ, σ = 3.4 Å and ϵ = 0.24037 kcal/mol
    baked in), then ASR! (asr.jl:3-17) and apply_tols! (ifc.jl:12).  None when
    oracle/_ref is not built."""
    h2 = _ref_lj_kernel("ref_H2_exec_LJ")
    if h2 is None:
        return None
    pairs, N = _lj_pairs_ad(pos, box, r_cut)
    n = 3 * N
    ifc2 = np.zeros((n, n), order="F")
    blk = np.zeros(9)
    for i, j, r in pairs:
        h2(_pd(r), _pd(blk))
        b = -blk.reshape((3, 3), order="F")
        ifc2[3 * i:3 * i + 3, 3 * j:3 * j + 3] = b
        ifc2[3 * j:3 * j + 3, 3 * i:3 * i + 3] = b
    for i in range(N):
        for a in range(3):
            for c in range(3):
                ifc2[3 * i + a, 3 * i + c] = -np.sum(ifc2[3 * i + a, c::3])
    ifc2[np.abs(ifc2) < tol] = 0.0
    return ifc2


def third_order_lj_ad_ref(pos, box, r_cut, tol):
    """third_order! with the AutoDiffCalculator for LJ
    (src/autodiff/third_order_AD.jl:1-69) driven by the reference's own
    generated third-derivative kernel (H3_exec_LJ): per pair i < j the block
    -H3(r_ij) is assigned at (i,i,j), (i,j,i), (j,i,i) and its negative at
    (i,j,j), (j,j,i), (j,i,j); then ASR! (asr.jl:19-40: every (iα, jβ, iγ)
    becomes minus the sum of its row over the third index) and apply_tols!
    (ifc.jl:30).  None when oracle/_ref is not built."""
    h3 = _ref_lj_kernel("ref_H3_exec_LJ")
    if h3 is None:
        return None
    pairs, N = _lj_pairs_ad(pos, box, r_cut)
    n = 3 * N
    psi = np.zeros((n, n, n), order="F")
    blk = np.zeros(27)
    for i, j, r in pairs:
        h3(_pd(r), _pd(blk))
        b = -blk.reshape((3, 3, 3), order="F")
        I, J = slice(3 * i, 3 * i + 3), slice(3 * j, 3 * j + 3)
        psi[I, I, J] = b
        psi[I, J, I] = b
        psi[J, I, I] = b
        psi[I, J, J] = -b
        psi[J, J, I] = -b
        psi[J, I, J] = -b
    six = psi.reshape((3, N, 3, N, 3, N), order="F")
    for i in range(N):
        six[:, i, :, :, :, i] = 0.0
        six[:, i, :, :, :, i] = -np.sum(six[:, i, :, :, :, :], axis=4)
    psi[np.abs(psi) < tol] = 0.0
    return psi


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


# ------------------------------------------------------------------ adjoint
def mcc3_loss_lj(pos, box, sigma, eps, r_cut, masses, phi, W, tol=1e-12):
    """L = Σ W·K3 in FP64 along the reference path (third_order → mass weight
    → mcc3 over modes [0, M)); used for central finite differences."""
    psi = third_order_lj(pos, box, sigma, eps, r_cut, tol)
    mw = mass_weight_third_order(psi, masses)
    M = W.shape[0]
    return float(np.sum(W * mcc3(mw, phi, modes=(0, M))))


def _lj_rad(r, sg, ep):
    """Φ′..Φ⁗ (LennardJones.jl:38-56) and the σ-derivatives of Φ′..Φ‴."""
    d1 = -ep * (48 * sg ** 12 / r ** 13 - 24 * sg ** 6 / r ** 7)
    d2 = 4 * ep * (156 * sg ** 12 / r ** 14 - 42 * sg ** 6 / r ** 8)
    d3 = -4 * ep * (2184 * sg ** 12 / r ** 15 - 336 * sg ** 6 / r ** 9)
    d4 = 4 * ep * (32760 * sg ** 12 / r ** 16 - 3024 * sg ** 6 / r ** 10)
    s1 = -ep * (576 * sg ** 11 / r ** 13 - 144 * sg ** 5 / r ** 7)
    s2 = 4 * ep * (1872 * sg ** 11 / r ** 14 - 252 * sg ** 5 / r ** 8)
    s3 = -4 * ep * (26208 * sg ** 11 / r ** 15 - 2016 * sg ** 5 / r ** 9)
    return d1, d2, d3, d4, s1, s2, s3


def _phi3_t(f1, f2, f3, nh, r):
    """ϕ₃ tensor (third_order_analytical.jl:216-224) from radial derivatives."""
    A = f3 - 3 * f2 / r + 3 * f1 / r ** 2
    B = (f2 - f1 / r) / r
    I = np.eye(3)
    return (np.einsum('a,b,c->abc', nh, nh, nh) * A +
            B * (np.einsum('bc,a->abc', I, nh) + np.einsum('ca,b->abc', I, nh) + np.einsum('ab,c->abc', I, nh)))


def _phi4_t(d1, d2, d3, d4, nh, r):
    """ϕ₄ tensor (fourth_order_analytical.jl:184-198)."""
    I = np.eye(3)
    E4 = d4 - 6 * d3 / r + 15 * d2 / r ** 2 - 15 * d1 / r ** 3
    E3 = (d3 - 3 * d2 / r + 3 * d1 / r ** 2) / r
    E2 = (d2 - d1 / r) / r ** 2
    nn = np.einsum('a,b->ab', nh, nh)
    v = sum(np.einsum(s, nn, I) for s in ['ab,cd->abcd', 'ac,bd->abcd', 'ad,bc->abcd',
                                             'bc,ad->abcd', 'bd,ac->abcd', 'cd,ab->abcd'])
    dd = np.einsum('ab,cd->abcd', I, I) + np.einsum('ac,bd->abcd', I, I) + np.einsum('ad,bc->abcd', I, I)
    return np.einsum('a,b,c,d->abcd', nh, nh, nh, nh) * E4 + v * E3 + dd * E2


def lj_adjoint(pos, box, sigma, eps, r_cut, masses, phi, W):
    """FP64 gradient of L = Σ W·K3 by the pair form of the chain rule:
    G = W ×₁φᵀ ×₂φᵀ ×₃φᵀ, C_AB = G'[AAA] − G'[AAB] − G'[ABA] − G'[BAA],
    ∂L/∂r_A = Σ_B ϕ₄(d_AB)·C_AB − Σ_B ϕ₄(d_BA)·C_BA, ∂L/∂ε = L/ε,
    ∂L/∂σ = Σ (∂ϕ₃/∂σ)·C.  Returns (dpos (N,3), dsigma, deps, L)."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    N = pos.shape[0]
    M = W.shape[0]
    ph = np.asarray(phi, dtype=np.float64)[:, :M]
    G = np.einsum('abc,ia,jb,kc->ijk', np.asarray(W, dtype=np.float64), ph, ph, ph)
    m = np.repeat(np.asarray(masses, dtype=np.float64), 3)
    Gp = G / np.sqrt(m[:, None, None] * m[None, :, None] * m[None, None, :])
    grad = np.zeros((N, 3))
    dsg = 0.0
    L = 0.0
    for A in range(N):
        for B in range(N):
            if A == B:
                continue
            r = np.array(pos[A] - pos[B])
            oracle_r = r.copy()
            lib().oracle_nearest_mirror(_pd(oracle_r), _pd(np.ascontiguousarray(box, dtype=np.float64)))
            rn = np.sqrt(oracle_r @ oracle_r)
            if not rn < r_cut:
                continue
            nh = oracle_r / rn
            d1, d2, d3, d4, s1, s2, s3 = _lj_rad(rn, sigma, eps)
            a, b = slice(3 * A, 3 * A + 3), slice(3 * B, 3 * B + 3)
            C = Gp[a, a, a] - Gp[a, a, b] - Gp[a, b, a] - Gp[b, a, a]
            L += np.sum(_phi3_t(d1, d2, d3, nh, rn) * C)
            dsg += np.sum(_phi3_t(s1, s2, s3, nh, rn) * C)
            v = np.einsum('abcd,abc->d', _phi4_t(d1, d2, d3, d4, nh, rn), C)
            grad[A] += v
            grad[B] -= v
    return grad, dsg, L / eps, L

"""Modal coupling constants mirroring ForceConstants.jl ``src/mcc.jl``.

* ``mcc3(psi, phi)``               mcc.jl:29-51 — result stays on the device
* ``mcc3(psi, phi, block_size)``   mcc.jl:89-120 — result is a host array
* ``mcc3_(psi, phi)``              mcc.jl:60-80 (``mcc3!``; Ψ is left intact here)
* ``mcc3_tens_opt(psi, phi)``      mcc.jl:11-20

``precision`` selects the arithmetic of the three mode products: "fp32" (FFMA,
the reference's Float32), "bf16x3" or "tf32x3" (split operands on the tensor
cores, FP32 accumulation).  ``modes=(lo, hi)`` restricts every mode axis to
φ[:, lo:hi] (0-based, half-open).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .arrays import as_julia, device_index, is_torch, julia_empty, ptr, stream_ptr


def _prep(psi, phi):
    psi = as_julia(psi, np.float32)
    phi = as_julia(phi, np.float32)
    n = int(phi.shape[0])
    if tuple(psi.shape) != (n, n, n) or tuple(phi.shape) != (n, n):
        raise ValueError("Ψ must be n×n×n and φ n×n")
    return psi, phi, n


def mcc3(psi, phi, block_size: int | None = None, precision: str = "fp32", modes=None):
    psi, phi, n = _prep(psi, phi)
    prec = _lib.PRECISIONS[precision]
    dev = device_index(psi) if is_torch(psi) else device_index(phi)
    if block_size is not None and not (block_size > 0 and n % block_size == 0):
        raise AssertionError("size(phi)[1] % block_size == 0")  # mcc.jl:91-92
    h = _lib.handle(dev)
    if block_size is not None:
        out = np.empty((n, n, n), dtype=np.float32, order="F")
        _lib.check(_lib.lib().fcb200_mcc3_blocked(h, ptr(psi), ptr(phi), n, int(block_size), prec, ptr(out),
                                                  stream_ptr(psi)))
        return out
    lo, hi = (0, n) if modes is None else (int(modes[0]), int(modes[1]))
    M = hi - lo
    device = f"cuda:{dev}" if (is_torch(psi) and psi.is_cuda) else "cpu"
    if device == "cpu" and is_torch(phi) and phi.is_cuda:
        device = f"cuda:{dev}"
    out = julia_empty((M, M, M), np.float32, device)
    _lib.check(_lib.lib().fcb200_mcc3(h, ptr(psi), ptr(phi), n, lo, hi, lo, hi, lo, hi, prec, ptr(out),
                                      stream_ptr(psi) or stream_ptr(phi)))
    return out


def mcc3_(psi, phi, precision: str = "fp32"):
    """``mcc3!``: the reference overwrites Ψ as scratch; here Ψ is left intact
    (the intermediates live in library scratch) and K3 is returned."""
    return mcc3(psi, phi, precision=precision)


def mcc3_tens_opt(psi, phi, precision: str = "fp32"):
    return mcc3(psi, phi, precision=precision)


def mcc3_window(psi, phi, n_range, m_range, l_range, precision: str = "fp32"):
    """One block of mcc3_blocked! (mcc.jl:123-134): K3 over three mode windows."""
    psi, phi, n = _prep(psi, phi)
    prec = _lib.PRECISIONS[precision]
    dev = device_index(psi) if is_torch(psi) else device_index(phi)
    shape = (n_range[1] - n_range[0], m_range[1] - m_range[0], l_range[1] - l_range[0])
    device = f"cuda:{dev}" if (is_torch(psi) and psi.is_cuda) else "cpu"
    out = julia_empty(shape, np.float32, device)
    _lib.check(_lib.lib().fcb200_mcc3(_lib.handle(dev), ptr(psi), ptr(phi), n, n_range[0], n_range[1],
                                      m_range[0], m_range[1], l_range[0], l_range[1], prec, ptr(out),
                                      stream_ptr(psi)))
    return out


def snapshot_lj(sys, pot, calc, phi, precision: str = "bf16x3", modes=None, psi_out=None, k3_out=None,
                stream: int = 0, dense: bool = False, packed: bool = False):
    """Fused third_order → mass_weight_third_order! → Float32 → mcc3 for one
    snapshot (LJ, or Stillinger-Weber when ``pot`` is a
    StillingerWeberSilicon), without the host round trip.  Buffers may be host
    or device; returns (psi_out, k3_out).  For LJ with a split precision the
    first two mode products use the block sparsity of Ψ unless ``dense``.
    With ``packed`` the K3 output holds only the entries p <= q <= s
    (``unpack_k3`` restores the full tensor)."""
    from .types import StillingerWeberSilicon
    n = 3 * sys.n_atoms
    lo, hi = (0, n) if modes is None else (int(modes[0]), int(modes[1]))
    M = hi - lo
    if k3_out is None:
        where = "cuda" if is_torch(phi) and phi.is_cuda else "cpu"
        k3_out = julia_empty((packed_k3_count(M),) if packed else (M, M, M), np.float32, where)
    dev = device_index(phi) if is_torch(phi) else 0
    flags = _lib.FCB_K3_PACKED if packed else 0
    if isinstance(pot, StillingerWeberSilicon):
        c0 = np.array([-0.333333333333, float(pot.cos0)], dtype=np.float64)
        _lib.check(_lib.lib().fcb200_snapshot_sw(
            _lib.handle(dev), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(calc.r_cut),
            float(calc.tol), ptr(c0), ptr(sys.masses), ptr(phi), lo, hi, _lib.PRECISIONS[precision] | flags,
            ptr(psi_out), ptr(k3_out), stream or stream_ptr(k3_out)))
        return psi_out, k3_out
    _lib.check(_lib.lib().fcb200_snapshot_lj(
        _lib.handle(dev), ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes), float(pot.sigma), float(pot.eps),
        float(calc.r_cut), float(calc.tol), ptr(sys.masses), ptr(phi), lo, hi,
        _lib.PRECISIONS[precision] | (_lib.FCB_MCC3_FORCE_DENSE if dense else 0) | flags,
        ptr(psi_out), ptr(k3_out), stream or stream_ptr(k3_out)))
    return psi_out, k3_out


def set_neighbour_capacity(cap: int, device: int = 0):
    """Fixes the neighbour capacity of the block-sparse snapshot path on this
    device's handle (fcb200_set_neighbour_capacity): 0 restores the default
    (one read-back of the largest neighbour count per snapshot_lj call);
    cap > 0 removes that read-back, so that the call can be captured in a CUDA
    graph, and an atom with more neighbours makes the next synchronize raise."""
    _lib.check(_lib.lib().fcb200_set_neighbour_capacity(_lib.handle(device), int(cap)))


def packed_k3_count(M: int) -> int:
    """Entries K3[p,q,s] with p <= q <= s of an M-mode K3 (FCB_K3_PACKED)."""
    return M * (M + 1) * (M + 2) // 6


def packed_k3_index(M: int):
    """Flat column-major index p + M(q + M s) of the full K3 for every packed
    position (entry (p,q,s), p <= q <= s, at s(s+1)(s+2)/6 + q(q+1)/2 + p)."""
    s = np.repeat(np.arange(M), [(x + 1) * (x + 2) // 2 for x in range(M)])
    q = np.concatenate([np.repeat(np.arange(x + 1), np.arange(1, x + 2)) for x in range(M)])
    base = s * (s + 1) * (s + 2) // 6 + q * (q + 1) // 2
    p = np.arange(packed_k3_count(M)) - base
    return p + M * (q + M * s)


def unpack_k3(packed, M: int) -> np.ndarray:
    """The full symmetric K3 (M×M×M, column-major) from its packed entries."""
    vals = np.asarray(packed.cpu() if is_torch(packed) else packed, dtype=np.float32).reshape(-1)
    idx = packed_k3_index(M)
    p, rest = idx % M, idx // M
    q, s = rest % M, rest // M
    out = np.empty((M, M, M), dtype=np.float32, order="F")
    for a, b, c in ((p, q, s), (p, s, q), (q, p, s), (q, s, p), (s, p, q), (s, q, p)):
        out[a, b, c] = vals
    return out

"""Buffers handed to the C ABI: numpy arrays (host) or torch tensors (device).

Dense tensors use Julia's column-major layout: element [i, j, k] at
i + n*(j + n*k).  Host results are Fortran-ordered numpy arrays; device results
are torch tensors whose strides are (1, n, n²), so t[i, j, k] has the same
meaning as the reference's Ψ[i+1, j+1, k+1].
"""
from __future__ import annotations

import numpy as np


def _torch():
    import torch
    return torch


def is_torch(x) -> bool:
    try:
        torch = _torch()
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


def ptr(x) -> int:
    if x is None:
        return 0
    if is_torch(x):
        return int(x.data_ptr())
    return int(x.ctypes.data)


def julia_empty(shape, dtype, device: str):
    """Uninitialised column-major array of `shape` on the host or a CUDA device."""
    size = int(np.prod(shape))
    if device == "cpu":
        return np.empty(shape, dtype=dtype, order="F")
    torch = _torch()
    tdt = {np.float64: torch.float64, np.float32: torch.float32}[np.dtype(dtype).type]
    flat = torch.empty(size, dtype=tdt, device=device)
    strides, s = [], 1
    for d in shape:
        strides.append(s)
        s *= d
    return flat.as_strided(tuple(shape), tuple(strides))


def as_julia(x, dtype):
    """Column-major contiguous version of x (no copy when already so)."""
    if is_torch(x):
        torch = _torch()
        tdt = {np.float64: torch.float64, np.float32: torch.float32}[np.dtype(dtype).type]
        x = x.to(tdt)
        dims = list(range(x.dim()))[::-1]
        if not x.permute(*dims).is_contiguous():
            x = x.permute(*dims).contiguous().permute(*dims)
        return x
    return np.asfortranarray(x, dtype=dtype)


def device_of(x) -> str:
    if is_torch(x) and x.is_cuda:
        return str(x.device)
    return "cpu"


def device_index(x) -> int:
    if is_torch(x) and x.is_cuda:
        return int(x.device.index or 0)
    return 0


def stream_ptr(x) -> int:
    """The caller's current torch stream for a device tensor (0 for host)."""
    if is_torch(x) and x.is_cuda:
        torch = _torch()
        return int(torch.cuda.current_stream(x.device).cuda_stream)
    return 0

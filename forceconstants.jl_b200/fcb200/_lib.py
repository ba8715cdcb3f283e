"""ctypes binding of ``libfcb200.so`` (the C ABI declared in ``include/fcb200.h``).

The shared library must exist in this directory (built by ``build.py``).  There
is no fallback: if it is missing, importing the compute entry points raises.
"""
from __future__ import annotations

import atexit
import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libfcb200.so")

FCB_OK = 0
FCB_ERR_ARG = 1
FCB_ERR_CUTOFF = 2
FCB_ERR_OOM = 3
FCB_ERR_CUDA = 4
FCB_ERR_TIMEOUT = 5
FCB_ERR_UNSUPPORTED = 6
FCB_ERR_BLOCK = 7

FCB_MCC3_FP32 = 0
FCB_MCC3_BF16X3 = 1
FCB_MCC3_TF32X3 = 2
FCB_ADJOINT_FP64 = 3
FCB_MCC3_FORCE_DENSE = 0x100
FCB_K3_PACKED = 0x200
PRECISIONS = {"fp32": FCB_MCC3_FP32, "bf16x3": FCB_MCC3_BF16X3, "tf32x3": FCB_MCC3_TF32X3}
# The adjoint also forms G in FP64 (FCB_ADJOINT_FP64).
ADJOINT_PRECISIONS = dict(PRECISIONS, fp64=FCB_ADJOINT_FP64)

FCB_PSI_MASS_WEIGHTED = 1

# Every symbol the header declares, with (restype, argtypes).
_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_I = ctypes.c_int
SIGNATURES = {
    "fcb200_version": (_I, []),
    "fcb200_last_error": (_I, [ctypes.c_char_p, ctypes.c_size_t]),
    "fcb200_create": (_I, [ctypes.POINTER(_P), _I]),
    "fcb200_destroy": (_I, [_P]),
    "fcb200_trim": (_I, [_P]),
    "fcb200_synchronize": (_I, [_P, _P]),
    "fcb200_set_wait_limit": (_I, [_P, _I64]),
    "fcb200_set_neighbour_capacity": (_I, [_P, _I]),
    "fcb200_third_order_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _D, _P, _P, _P, _I, _P]),
    "fcb200_mass_weight3": (_I, [_P, _P, _P, _I64, _P]),
    "fcb200_second_order_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _D, _P, _P, _P]),
    "fcb200_get_modes": (_I, [_P, _P, _I64, _I, _P, _P, _P, _P]),
    "fcb200_fd_third_order_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _P, _I64, _D, _P, _P]),
    "fcb200_fd_third_order_sw": (_I, [_P, _P, _I64, _P, _P, _I64, _D, _P, _P]),
    "fcb200_fd_second_order_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _D, _D, _D, _P, _P]),
    "fcb200_fd_second_order_sw": (_I, [_P, _P, _I64, _P, _D, _D, _D, _P, _P]),
    "fcb200_mcc3": (_I, [_P, _P, _P, _I64, _I64, _I64, _I64, _I64, _I64, _I64, _I, _P, _P]),
    "fcb200_mcc3_blocked": (_I, [_P, _P, _P, _I64, _I64, _I, _P, _P]),
    "fcb200_snapshot_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _D, _P, _P, _I64, _I64, _I, _P, _P, _P]),
    "fcb200_set_profiling": (_I, [_P, _I]),
    "fcb200_phase_times": (_I, [_P, ctypes.POINTER(_D), _I]),
    "fcb200_third_order_lj_noalloc": (_I, [_P, _I64, _P, _D, _D, _D, _D, _P, _P, _P, _I, _P]),
    "fcb200_third_order_sw": (_I, [_P, _P, _I64, _P, _D, _D, _P, _P, _P, _P, _I, _P]),
    "fcb200_second_order_sw": (_I, [_P, _P, _I64, _P, _D, _D, _P, _P, _P, _P]),
    "fcb200_snapshot_sw": (_I, [_P, _P, _I64, _P, _D, _D, _P, _P, _P, _I64, _I64, _I, _P, _P, _P]),
    "fcb200_autotune_mcc3": (_I, [_P, _I64, _I, ctypes.c_char_p, _P]),
    "fcb200_batch_create": (_I, [_P, _I, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "fcb200_batch_add_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _D, _P, _P, _P]),
    "fcb200_batch_set_positions": (_I, [_P, _I64, _P, _P]),
    "fcb200_batch_run": (_I, [_P, _P]),
    "fcb200_batch_info": (_I, [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                               ctypes.POINTER(ctypes.c_size_t)]),
    "fcb200_batch_lane": (_I, [_P, _I64, ctypes.POINTER(_I64)]),
    "fcb200_batch_destroy": (_I, [_P]),
    "fcb200_mcc3_adjoint_lj": (_I, [_P, _P, _I64, _P, _D, _D, _D, _P, _P, _I64, _P, _I, _P,
                                    ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D), _P]),
}

_lib = None


class FCB200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fcb200 error {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
                " (there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> tuple[int, str]:
    buf = ctypes.create_string_buffer(1024)
    code = lib().fcb200_last_error(buf, len(buf))
    return code, buf.value.decode(errors="replace")


def check(status: int) -> None:
    """Map a status to the reference's error behaviour.

    The reference's ``@assert``s (cutoff vs box, block size divisibility)
    become ``AssertionError`` with the reference's message; everything else is
    an ``FCB200Error``.
    """
    if status == FCB_OK:
        return
    code, msg = last_error()
    if status == FCB_ERR_CUTOFF:
        raise AssertionError(msg if "SW" in msg else "Cutoff larger than L/2")
    if status == FCB_ERR_BLOCK:
        raise AssertionError("size(phi)[1] % block_size == 0")
    raise FCB200Error(status, msg)


_handles: dict[int, int] = {}


def handle(device: int = 0) -> int:
    """Lazily created library handle per CUDA device (owns cached scratch)."""
    h = _handles.get(device)
    if h is None:
        out = _P()
        check(lib().fcb200_create(ctypes.byref(out), device))
        h = out.value
        _handles[device] = h
    return h


@atexit.register
def _release_handles() -> None:
    if _lib is None:
        return
    for h in list(_handles.values()):
        _lib.fcb200_destroy(h)
    _handles.clear()

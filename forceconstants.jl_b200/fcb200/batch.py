"""Batches of LJ snapshots through the C ABI (fcb200_batch_*): IFC3 assembly,
mass weighting and full-mode mcc3 for many snapshots, replayed as one CUDA
graph after the first (eager) run."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .arrays import julia_empty, ptr


class SnapshotBatch:
    def __init__(self, precision: str = "bf16x3", hbm_budget_bytes: int = 0, device: int = 0):
        self.device = device
        self._h = _lib.handle(device)
        out = ctypes.c_void_p()
        _lib.check(_lib.lib().fcb200_batch_create(self._h, _lib.PRECISIONS[precision], int(hbm_budget_bytes),
                                                  ctypes.byref(out)))
        self._b = out.value
        self.k3 = []

    def add(self, sys, pot, calc, phi, k3_out=None):
        """Adds one snapshot; returns its K3 device tensor (written by run())."""
        n = 3 * sys.n_atoms
        if k3_out is None:
            k3_out = julia_empty((n, n, n), np.float32, f"cuda:{self.device}")
        phi = np.asfortranarray(np.asarray(phi, dtype=np.float32))
        _lib.check(_lib.lib().fcb200_batch_add_lj(self._b, ptr(sys.positions), sys.n_atoms, ptr(sys.box_sizes),
                                                  float(pot.sigma), float(pot.eps), float(calc.r_cut),
                                                  float(calc.tol), ptr(sys.masses), ptr(phi), ptr(k3_out)))
        self.k3.append(k3_out)
        return k3_out

    def set_positions(self, index: int, positions, stream: int = 0):
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        _lib.check(_lib.lib().fcb200_batch_set_positions(self._b, int(index), ptr(pos), stream))

    def run(self, stream: int = 0):
        _lib.check(_lib.lib().fcb200_batch_run(self._b, stream))

    def info(self):
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        d = ctypes.c_size_t()
        _lib.check(_lib.lib().fcb200_batch_info(self._b, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                ctypes.byref(d)))
        return {"snapshots": a.value, "lanes": b.value, "graph_nodes": c.value, "scratch_bytes": d.value}

    def lane(self, index: int) -> int:
        """Lane of snapshot ``index`` in the current plan (after the first run)."""
        out = ctypes.c_int64()
        _lib.check(_lib.lib().fcb200_batch_lane(self._b, int(index), ctypes.byref(out)))
        return out.value

    def close(self):
        if self._b:
            _lib.lib().fcb200_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_mcc3(n: int, precision: str = "bf16x3", cache_path: str | None = None, device: int = 0):
    _lib.check(_lib.lib().fcb200_autotune_mcc3(_lib.handle(device), int(n), _lib.PRECISIONS[precision],
                                               cache_path.encode() if cache_path else None, 0))

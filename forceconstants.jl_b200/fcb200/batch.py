"""Batches of LJ snapshots through the C ABI (fcb200_batch_*): IFC3 assembly,
mass weighting and full-mode mcc3 for many snapshots, replayed as one CUDA
graph after the first (eager) run; and trajectory_k3, which feeds the frames of
an MD trajectory (io.jl:319-353's xyz format) through such a batch."""
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


def trajectory_k3(path: str, n_atoms: int, n_steps: int, box_sizes, masses, pot, calc, phi,
                  precision: str = "bf16x3", frames_per_batch: int = 8, on_frame=None, device: int = 0):
    """MD trajectory in, K3 out.  The frames of the xyz trajectory at `path`
    (parse_xyz, io.jl:319-353: positions in file order, one cell, masses and
    modes φ shared by every frame) run through one SnapshotBatch of
    `frames_per_batch` snapshots; each further group of frames replaces the
    snapshots' positions (fcb200_batch_set_positions) and replays the same
    CUDA graph.  on_frame(step, ids, k3) receives every frame's K3 as a device
    tensor, in frame order, before the next group overwrites it; without
    on_frame the K3 of every frame comes back as a host array, in a list.
    Frames the file does not hold (parse_xyz leaves them empty) are skipped."""
    import torch
    from .io import parse_xyz
    from .types import SuperCellSystem
    if frames_per_batch < 1:
        raise ValueError("frames_per_batch must be at least 1")
    positions, ids = parse_xyz(path, n_atoms, n_steps)
    frames = [t for t in range(n_steps) if positions[t].shape[0] == n_atoms]
    out = []
    if not frames:
        return out
    phi = np.asfortranarray(np.asarray(phi, dtype=np.float32))
    masses = np.asarray(masses, dtype=np.float64)
    nslots = min(frames_per_batch, len(frames))
    batch = SnapshotBatch(precision, device=device)
    try:
        slots = [batch.add(SuperCellSystem(positions[t], masses, box_sizes), pot, calc, phi)
                 for t in frames[:nslots]]
        for g0 in range(0, len(frames), nslots):
            group = frames[g0:g0 + nslots]
            if g0:
                for i, t in enumerate(group):
                    batch.set_positions(i, positions[t])
            batch.run()
            torch.cuda.synchronize(device)
            for i, t in enumerate(group):
                if on_frame is not None:
                    on_frame(t, ids[t], slots[i])
                else:
                    out.append(slots[i].cpu().numpy())
    finally:
        batch.close()
    return out


def autotune_mcc3(n: int, precision: str = "bf16x3", cache_path: str | None = None, device: int = 0):
    _lib.check(_lib.lib().fcb200_autotune_mcc3(_lib.handle(device), int(n), _lib.PRECISIONS[precision],
                                               cache_path.encode() if cache_path else None, 0))

"""Crystal builders standing in for SimpleCrystals.jl (``FCC``, ``Diamond``).

Atoms are ordered cell by cell (x outer, then y, then z) and, inside a
conventional cell, in the basis order below.  The FCC basis order puts atom 2 at
(a/2, a/2, 0), which is what the reference's known-answer values in
``test/runtests.jl:109-136`` imply; the box is the bounding box (types.jl:39).
"""
from __future__ import annotations

import numpy as np

from .types import SuperCellSystem

ATOMIC_MASS = {"Ar": 39.95, "Si": 28.0855}

FCC_BASIS = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
DIAMOND_BASIS = np.vstack([FCC_BASIS, FCC_BASIS + 0.25])


def _lattice(a: float, basis: np.ndarray, cells) -> tuple[np.ndarray, np.ndarray]:
    nx, ny, nz = (int(c) for c in cells)
    pos = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                for b in basis:
                    pos.append((np.array([i, j, k], dtype=np.float64) + b) * a)
    box = np.array([nx * a, ny * a, nz * a], dtype=np.float64)
    return np.array(pos, dtype=np.float64), box


def FCC(a: float, element: str = "Ar", cells=(4, 4, 4)) -> SuperCellSystem:
    pos, box = _lattice(a, FCC_BASIS, cells)
    return SuperCellSystem(pos, np.full(len(pos), ATOMIC_MASS.get(element, 1.0)), box)


def Diamond(a: float, element: str = "Si", cells=(3, 3, 3)) -> SuperCellSystem:
    pos, box = _lattice(a, DIAMOND_BASIS, cells)
    return SuperCellSystem(pos, np.full(len(pos), ATOMIC_MASS.get(element, 1.0)), box)


def displaced(sys: SuperCellSystem, std: float, seed: int) -> SuperCellSystem:
    """i.i.d. Gaussian displacement of every Cartesian component (seeded)."""
    rng = np.random.default_rng(seed)
    return SuperCellSystem(sys.positions + rng.normal(0.0, std, size=sys.positions.shape), sys.masses.copy(),
                           sys.box_sizes.copy(), sys.length_unit, sys.mass_unit)

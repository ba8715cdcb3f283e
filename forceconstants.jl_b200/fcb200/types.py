"""Data model mirroring ForceConstants.jl ``src/types.jl`` and the potentials.

* ``SuperCellSystem``       types.jl:20-50 (positions, masses, orthorhombic box)
* ``LJ``                    interactions/LennardJones.jl:6-23
* ``StillingerWeberSilicon`` interactions/SW.jl:3-44 (LAMMPS Si.sw parameters)
* ``AnalyticalCalculator`` / ``AutoDiffCalculator``  types.jl:191-201
* ``DenseForceConstants``   types.jl:76-90 (``.values``, ``.units``, ``.tol``)

Units are carried as strings (the reference uses Unitful); numbers are in the
potential's units: LJ in (σ, ϵ) units, SW in eV and Å.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class SuperCellSystem:
    positions: np.ndarray          # (N, 3) float64
    masses: np.ndarray             # (N,)   float64 (amu)
    box_sizes: np.ndarray          # (3,)   float64
    length_unit: str = "Å"
    mass_unit: str = "u"

    def __post_init__(self):
        self.positions = np.ascontiguousarray(np.asarray(self.positions, dtype=np.float64).reshape(-1, 3))
        self.masses = np.ascontiguousarray(np.asarray(self.masses, dtype=np.float64).reshape(-1))
        self.box_sizes = np.ascontiguousarray(np.asarray(self.box_sizes, dtype=np.float64).reshape(3))
        if self.masses.shape[0] != self.positions.shape[0]:
            raise ValueError("one mass per atom is required")

    @property
    def n_atoms(self) -> int:
        return int(self.positions.shape[0])

    def volume(self) -> float:
        return float(np.prod(self.box_sizes))


def n_atoms(sys: SuperCellSystem) -> int:
    return sys.n_atoms


def masses(sys: SuperCellSystem) -> np.ndarray:
    return sys.masses


def positions(sys: SuperCellSystem) -> np.ndarray:
    return sys.positions


class Potential:
    pass


class PairPotential(Potential):
    pass


class ThreeBodyPotential(Potential):
    pass


@dataclass
class LJ(PairPotential):
    """12-6 Lennard-Jones, LennardJones.jl:6-23."""
    sigma: float
    eps: float
    r_cut: float
    energy_unit: str = "kcal mol^-1"
    length_unit: str = "Å"

    def potential(self, r):
        k = (self.sigma / r) ** 6
        return 4 * self.eps * k * (k - 1)


@dataclass
class StillingerWeberSilicon(ThreeBodyPotential):
    """SW.jl:29-44 with the LAMMPS Si.sw parameters (eV, Å)."""
    eps: float = 2.1683
    sigma: float = 2.0951
    a: float = 1.80
    lam: float = 21.0
    gamma: float = 1.20
    cos0: float = -1.0 / 3.0
    A: float = 7.049556277
    B: float = 0.6022245584
    p: float = 4.0
    q: float = 0.0
    energy_unit: str = "eV"
    length_unit: str = "Å"

    @property
    def r_cut(self) -> float:
        return self.a * self.sigma

    @property
    def gamma_sigma(self) -> float:
        return self.sigma * self.gamma

    @property
    def lambda_epsilon(self) -> float:
        return self.eps * self.lam


class ForceConstantCalculator:
    pass


@dataclass
class AnalyticalCalculator(ForceConstantCalculator):
    tol: float
    r_cut: float


@dataclass
class AutoDiffCalculator(ForceConstantCalculator):
    tol: float
    r_cut: float


FD_STEP = 0.04 * 0.5291772109   # the reference's default h: 0.04 bohr in Å (types.jl:209)


@dataclass
class FiniteDiffCalculator(ForceConstantCalculator):
    """types.jl:203-213: (tol, r_cut; h)."""
    tol: float
    r_cut: float
    h: float = FD_STEP


@dataclass
class DenseForceConstants:
    """types.jl:76-80.  ``values`` is a numpy array (host) or a torch tensor
    (device) with Julia's column-major index semantics: values[i, j, k] is
    Ψ[i+1, j+1, k+1] of the reference."""
    values: object
    units: str
    tol: float

    def __getitem__(self, idx):
        return self.values[idx]

    @property
    def shape(self):
        return tuple(self.values.shape)

    def size(self):
        return self.shape

    def n_modes(self) -> int:
        return self.shape[0]


def energy_unit(pot) -> str:
    return pot.energy_unit


def length_unit(pot) -> str:
    return pot.length_unit

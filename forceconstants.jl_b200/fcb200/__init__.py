"""fcb200 — B200-native third-order force constants and modal coupling constants.

Host-side mirror of the ForceConstants.jl API for its dense IFC3 + mcc3 path,
calling the C ABI of ``libfcb200.so`` (``include/fcb200.h``).
"""
from .batch import SnapshotBatch, trajectory_k3
from .crystals import FCC, Diamond, displaced
from .ifc import (asr_satisfied, dynamical_matrix, get_modes, mass_weight_third_order_, second_order,
                  second_order_, third_order, third_order_)
from .finite_diff import third_order_fd, third_order_finite_diff_eng
from .io import load_force_constants, load_third_order_txt, parse_xyz, save_second_order, save_third_order
from .mcc import (mcc3, mcc3_, mcc3_tens_opt, mcc3_window, packed_k3_count, set_neighbour_capacity, snapshot_lj,
                  unpack_k3)
from .types import (LJ, AnalyticalCalculator, AutoDiffCalculator, DenseForceConstants, FiniteDiffCalculator,
                    PairPotential, Potential,
                    StillingerWeberSilicon, SuperCellSystem, ThreeBodyPotential, energy_unit, length_unit, masses,
                    n_atoms, positions)

__all__ = [
    "FCC", "Diamond", "displaced", "asr_satisfied", "dynamical_matrix", "get_modes", "mass_weight_third_order_",
    "second_order", "second_order_", "third_order", "third_order_", "mcc3", "mcc3_", "mcc3_tens_opt",
    "mcc3_window", "snapshot_lj", "packed_k3_count", "unpack_k3", "LJ", "AnalyticalCalculator", "AutoDiffCalculator", "DenseForceConstants",
    "PairPotential", "Potential", "StillingerWeberSilicon", "SuperCellSystem", "ThreeBodyPotential",
    "energy_unit", "length_unit", "masses", "n_atoms", "positions", "parse_xyz", "save_third_order",
    "save_second_order", "load_third_order_txt", "load_force_constants", "FiniteDiffCalculator", "third_order_fd",
    "third_order_finite_diff_eng", "SnapshotBatch", "trajectory_k3",
    "set_neighbour_capacity",
]

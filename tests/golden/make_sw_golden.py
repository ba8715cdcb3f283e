"""SW golden fixtures from the reference's own derivative kernels.

Runs the Stillinger-Weber triplet loop (``oracle/sw_oracle.c``, restating
``src/autodiff/third_order_AD.jl:71-224`` and ``second_order_AD.jl:40-110``)
with the reference's machine-generated block kernels, translated from the
reference checkout into ``oracle/_ref/libswref.so`` by ``oracle/build.py``.
Writes ``sw_diamond_*.npz``: positions, box, IFC2 (dense) and IFC3 (sparse:
flat column-major indices + values), tol = 1e-12, r_cut = the SW cutoff aσ.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def diamond(a, cells):
    fcc = np.array([[0, 0, 0], [.5, .5, 0], [.5, 0, .5], [0, .5, .5]])
    basis = np.vstack([fcc, fcc + 0.25])
    pos = [(np.array([i, j, k]) + b) * a for i in range(cells[0]) for j in range(cells[1])
           for k in range(cells[2]) for b in basis]
    return np.array(pos), np.array(cells, dtype=float) * a


def main(reference_root: str) -> None:
    sys.path.insert(0, ROOT)
    from oracle.build import build_oracle, build_reference_translation
    build_oracle()
    if build_reference_translation(reference_root) is None:
        raise SystemExit("reference checkout not found: cannot build oracle/_ref/libswref.so")
    from oracle import oracle as O
    rc = O.lib().oracle_sw_rcut()
    cases = [("sw_diamond_1x1x1_std0.03_seed5", (1, 1, 1), 0.03, 5),
             ("sw_diamond_2x2x2_std0.03_seed7", (2, 2, 2), 0.03, 7)]
    for name, cells, std, seed in cases:
        pos, box = diamond(5.43, cells)
        pos = pos + np.random.default_rng(seed).normal(0.0, std, size=pos.shape)
        psi = O.third_order_sw(pos, box, rc, 1e-12, use_ref=True)
        ifc2 = O.second_order_sw(pos, box, rc, 1e-12, use_ref=True)
        flat = psi.reshape(-1, order="F")
        idx = np.flatnonzero(flat).astype(np.int64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), positions=pos, box=box, r_cut=rc, tol=1e-12,
                            ifc2=ifc2, ifc3_index=idx, ifc3_value=flat[idx], n=psi.shape[0],
                            source="reference generated SW kernels (translated), third_order_AD.jl:71-224")
        print(name, "nnz", idx.size)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} FORCECONSTANTS_JL_CHECKOUT")
    main(sys.argv[1])

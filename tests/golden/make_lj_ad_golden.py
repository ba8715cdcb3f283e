"""LJ golden fixture from the reference's own AutoDiffCalculator kernels.

Runs the LJ loops of the AutoDiffCalculator (``oracle.third_order_lj_ad_ref``
and ``oracle.second_order_lj_ad_ref``, restating
``src/autodiff/third_order_AD.jl:1-69`` and ``second_order_AD.jl:1-37``) with
the reference's machine-generated pair kernels ``H3_exec_LJ`` / ``H2_exec_LJ``,
translated from the reference checkout into ``oracle/_ref/libswref.so`` by
``oracle/build.py``.  Writes ``lj_ad_fcc_2x2x2_std0.05_seed3.npz``: positions,
box, IFC2 (dense) and IFC3 (sparse: flat column-major indices + values),
tol = 1e-12, r_cut = 8.5 Å, σ = 3.4 Å, ϵ = 0.24037 kcal/mol (the values baked
into the generated kernels).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
NAME = "lj_ad_fcc_2x2x2_std0.05_seed3"


def main(reference_root: str) -> None:
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "forceconstants.jl_b200"))
    from oracle.build import build_oracle, build_reference_translation
    build_oracle()
    if build_reference_translation(reference_root) is None:
        raise SystemExit("reference checkout not found: cannot build oracle/_ref/libswref.so")
    import fcb200
    from oracle import oracle as O
    s = fcb200.displaced(fcb200.FCC(5.2468, "Ar", (2, 2, 2)), 0.05, 3)
    psi = O.third_order_lj_ad_ref(s.positions, s.box_sizes, 8.5, 1e-12)
    ifc2 = O.second_order_lj_ad_ref(s.positions, s.box_sizes, 8.5, 1e-12)
    flat = psi.reshape(-1, order="F")
    idx = np.flatnonzero(flat).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, NAME + ".npz"), positions=s.positions, box=s.box_sizes, r_cut=8.5,
                        tol=1e-12, sigma=3.4, eps=0.24037, ifc2=ifc2, ifc3_index=idx, ifc3_value=flat[idx],
                        n=psi.shape[0],
                        source="reference generated LJ kernels (translated), third_order_AD.jl:1-69, "
                               "second_order_AD.jl:1-37")
    print(NAME, "nnz", idx.size)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} FORCECONSTANTS_JL_CHECKOUT")
    main(sys.argv[1])

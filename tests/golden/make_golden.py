"""Regenerate the committed golden fixtures under ``tests/golden/``.

1. ``lj_values.json`` — the known-answer values of the reference test-set
   "LJ Values" (ForceConstants.jl ``test/runtests.jl:109-136``), read as text
   from the reference's test file: 256-atom FCC argon (a = 5.2468 Å, 4×4×4),
   LJ σ = 3.4 Å, ϵ = 0.24037 kcal/mol, r_cut = 8.5 Å, tol = 1e-8.  Julia's
   ``≈`` is rtol = √eps(Float64) for these scalars.

2. ``sw_*.npz`` — Stillinger-Weber IFC2/IFC3 produced by the reference's own
   machine-generated derivative kernels (``src/autodiff/generated_derivatives``)
   translated to C by ``oracle/translate_sw_ref.py`` and driven by the
   reference triplet loop (``src/autodiff/third_order_AD.jl:71-224``) restated
   in ``oracle/sw_oracle.c``.  Stored sparsely (flat column-major index,
   value) because the dense tensors are mostly zeros.

Run from the repository root on a machine that has the reference checkout:
``python tests/golden/make_golden.py REFERENCE_ROOT`` (the ForceConstants.jl
checkout; required).
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def extract_lj_values(runtests_path: str) -> dict:
    text = open(runtests_path, encoding="utf-8").read()
    start = text.index('@testset "LJ Values"')
    end = text.index("end", text.index("ifc3[4,1,2]", start))
    block = text[start:end]
    out = {"ifc2": [], "ifc3": []}
    for m in re.finditer(r"@test\s+(ifc[23])\[([0-9, ]+)\]\s*≈\s*([-0-9.eE]+)", block):
        name, idx, val = m.group(1), m.group(2), float(m.group(3))
        out[name].append({"index_1based": [int(x) for x in idx.split(",")], "value": val})
    out["source"] = "ForceConstants.jl test/runtests.jl:109-136 (@testset \"LJ Values\")"
    out["system"] = {"lattice": "FCC", "a": 5.2468, "cells": [4, 4, 4], "sigma": 3.4,
                     "eps": 0.24037, "r_cut": 8.5, "tol": 1e-8, "units": "kcal/mol, Angstrom"}
    out["rtol"] = 1.4901161193847656e-08
    return out


def main(reference_root: str) -> None:
    lj = extract_lj_values(os.path.join(reference_root, "test", "runtests.jl"))
    with open(os.path.join(HERE, "lj_values.json"), "w") as f:
        json.dump(lj, f, indent=1)
    print("wrote lj_values.json:", len(lj["ifc2"]), "ifc2 +", len(lj["ifc3"]), "ifc3 values")
    sw_path = os.path.join(HERE, "make_sw_golden.py")
    if os.path.exists(sw_path):
        sys.path.insert(0, HERE)
        import make_sw_golden  # noqa: E402
        make_sw_golden.main(reference_root)
    if os.path.exists(os.path.join(HERE, "make_lj_ad_golden.py")):
        sys.path.insert(0, HERE)
        import make_lj_ad_golden  # noqa: E402
        make_lj_ad_golden.main(reference_root)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} FORCECONSTANTS_JL_CHECKOUT")
    main(sys.argv[1])

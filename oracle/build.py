"""ORACLE build recipe — test infrastructure only.

Compiles the CPU restatements under ``oracle/`` into ``oracle/liboracle.so``
(gcc, OpenMP, no fused multiply-add so that evaluation order is exactly the
order written in the C source).  When the ForceConstants.jl sources are present
on this machine, also translates the reference's machine-generated
Stillinger-Weber derivative kernels into C under ``oracle/_ref/`` and compiles
them into ``oracle/_ref/libswref.so`` (see ``oracle/translate_sw_ref.py``).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
SOURCES = ["lj_oracle.c", "sw_oracle.c", "fd_oracle.c"]
LIB = os.path.join(HERE, "liboracle.so")
CFLAGS = ["-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=c11"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES if os.path.exists(os.path.join(HERE, s))]
    if force or _stale(LIB, srcs):
        cmd = ["gcc", *CFLAGS, *srcs, "-o", LIB, "-lm"]
        subprocess.run(cmd, check=True)
    return LIB


def build_reference_translation(reference_root: str | None = None, force: bool = False) -> str | None:
    """Translate + compile the reference's generated SW and LJ derivative kernels.

    ``reference_root`` (or the environment variable FCB200_REFERENCE_ROOT) is
    the ForceConstants.jl checkout; there is no default.  Returns the path of
    ``oracle/_ref/libswref.so``, or None when no checkout is given or found and
    no previously built library exists.
    """
    if HERE not in sys.path:
        sys.path.append(HERE)
    from translate_sw_ref import translate_all  # noqa: E402  (sibling module)

    reference_root = reference_root or os.environ.get("FCB200_REFERENCE_ROOT")
    lib = os.path.join(REF_OUT, "libswref.so")
    gen_dir = os.path.join(reference_root, "src", "autodiff", "generated_derivatives") if reference_root else None
    if gen_dir is None or not os.path.isdir(gen_dir):
        return lib if os.path.exists(lib) else None
    os.makedirs(REF_OUT, exist_ok=True)
    c_path = os.path.join(REF_OUT, "sw_generated.c")
    deps = [os.path.join(HERE, "sw_oracle.c"), os.path.join(HERE, "lj_oracle.c")]
    if force or _stale(c_path, [os.path.join(HERE, "translate_sw_ref.py")]):
        translate_all(gen_dir, c_path)
    if force or _stale(lib, [c_path, *deps]):
        cmd = ["gcc", "-O1", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-DSW_BLOCKS_FROM_REFERENCE", *deps, c_path, "-o", lib, "-lm"]
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    print(build_oracle(force="--force" in sys.argv))
    roots = [a for a in sys.argv[1:] if not a.startswith("--")]
    print(build_reference_translation(roots[0] if roots else None, force="--force" in sys.argv))

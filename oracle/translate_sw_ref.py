"""ORACLE build step — test infrastructure only.

Translates ForceConstants.jl's machine-generated derivative kernels, read where
they lie in the reference checkout, into C for the CPU oracle.  Nothing here is
committed output: the generated C goes to ``oracle/_ref/`` (git-ignored) and is
compiled together with ``oracle/sw_oracle.c`` (built with
``-DSW_BLOCKS_FROM_REFERENCE``) into ``oracle/_ref/libswref.so``.

Inputs (relative to the reference root):

* ``src/autodiff/generated_derivatives/SW/H3_exec_{ij,iij,ijj,ikk,jjk,jkk,ijk}.jl``
  and ``SW/H2_exec_{pair,ij,ik,jk}.jl`` — FastDifferentiation output: one
  function per block, straight-line SSA statements
  ``var"##n" = a op b`` and ``result[CartesianIndex(a,b,c)] = v``.
  Used by ``third_order!``/``second_order!`` for SW
  (``src/autodiff/third_order_AD.jl:71-170``, ``second_order_AD.jl:40-110``).
* ``LJ/H2_exec_LJ.jl``, ``LJ/H3_exec_LJ.jl`` — FastDifferentiation output for
  the LJ pair (σ and ϵ of the reference's tests baked in), used by
  ``second_order!``/``third_order!`` with the AutoDiffCalculator
  (``second_order_AD.jl:1-37``, ``third_order_AD.jl:1-69``).
* ``SW_sym_iik/H3_exec_iik_{abc}.jl`` — Symbolics output, one prefix-form
  expression per component of the iik block.  The reference builds this block
  at run time with Symbolics from ``three_body_potential_nounits`` using the
  potential's exact cosθ₀ = -1/3 (``SW/H3_exec_iik.jl:1-44``, called at
  ``third_order_AD.jl:80,141``); these files hold the same expressions with the
  constant written as 0.333333333333, which is replaced by the exact value.

Julia semantics reproduced: left-to-right n-ary ``+``/``*``; ``x^2`` is
``x*x`` and ``x^3`` is ``x*x*x`` (Julia's integer-power special cases); other
powers use ``pow``; ``2var`` juxtaposition is multiplication.
"""
from __future__ import annotations

import os
import re

SW3 = ["ij", "iij", "ijj", "ikk", "jjk", "jkk", "ijk"]
SW2 = ["pair", "ij", "ik", "jk"]
EXACT_THIRD = "0.3333333333333333"

_num = r"-?(?:\d+\.\d*|\d*\.\d+|\d+)(?:[eE][-+]?\d+)?"
_var = r'var"##(\d+)"'
_inp = r"input_variables\[(\d+)\]"


def _term(t: str) -> str:
    t = t.strip()
    m = re.fullmatch(_var, t)
    if m:
        return f"v{m.group(1)}"
    m = re.fullmatch(_inp, t)
    if m:
        return f"x[{int(m.group(1)) - 1}]"
    m = re.fullmatch(rf"({_num}){_var}", t)          # juxtaposition: 2var"##5"
    if m:
        return f"({float(m.group(1))!r} * v{m.group(2)})"
    m = re.fullmatch(rf"({_num})\s*\*?\s*{_inp}", t)
    if m:
        return f"({float(m.group(1))!r} * x[{int(m.group(2)) - 1}])"
    if re.fullmatch(_num, t):
        return repr(float(t))
    raise ValueError(f"unrecognised term: {t!r}")


def _pow(a: str, b: str) -> str:
    try:
        e = float(b)
    except ValueError:
        return f"pow({a}, {b})"
    if e == 2.0:
        return f"({a} * {a})"
    if e == 3.0:
        return f"(({a} * {a}) * {a})"
    return f"pow({a}, {e!r})"


def _rhs(expr: str) -> str:
    e = expr.strip()
    m = re.fullmatch(r"(exp|sqrt|log|abs)\((.*)\)", e)
    if m:
        return f"{'fabs' if m.group(1) == 'abs' else m.group(1)}({_term(m.group(2))})"
    for op in [" + ", " - ", " * ", " / ", " ^ "]:
        if op in e:
            a, b = e.split(op, 1)
            a, b = _term(a), _term(b)
            if op == " ^ ":
                return _pow(a, b)
            return f"({a}{op}{b})"
    if e.startswith("-"):
        return f"(-{_term(e[1:])})"
    return _term(e)


def translate_fd(path: str, cname: str, cos0_exact: bool = False) -> str:
    """FastDifferentiation straight-line function → C function (x in, out[])."""
    lines = []
    for raw in open(path, encoding="utf-8"):
        s = raw.strip()
        if not s or s.startswith("#"):
            continue
        m = re.fullmatch(r'var"##(\d+)" = (.*)', s)
        if m:
            rhs = m.group(2)
            if cos0_exact:
                rhs = rhs.replace("0.333333333333", EXACT_THIRD)
            lines.append(f"    const double v{m.group(1)} = {_rhs(rhs)};")
            continue
        m = re.fullmatch(r"result\[CartesianIndex\(([\d, ]+)\)\] = (.*)", s)
        if m:
            idx = [int(t) - 1 for t in m.group(1).split(",")]
            flat = idx[0] + 3 * idx[1] + (9 * idx[2] if len(idx) == 3 else 0)
            lines.append(f"    out[{flat}] = {_term(m.group(2))};")
    return f"void {cname}(const double* x, double* out) {{\n" + "\n".join(lines) + "\n}\n"


class _Prefix:
    """Recursive-descent parser for Symbolics' prefix form, emitting SSA C."""

    def __init__(self, text: str):
        self.s = text
        self.i = 0
        self.out: list[str] = []
        self.k = 0

    def _ws(self):
        while self.i < len(self.s) and self.s[self.i] in " \n\t":
            self.i += 1

    def _tmp(self, expr: str) -> str:
        self.k += 1
        self.out.append(f"    const double t{self.k} = {expr};")
        return f"t{self.k}"

    def parse(self) -> str:
        self._ws()
        s = self.s
        if s.startswith("(", self.i):
            j = s.index(")", self.i)
            op = s[self.i + 1:j]
            self.i = j + 1
            assert s[self.i] == "(", s[self.i:self.i + 20]
            self.i += 1
            args = []
            while True:
                args.append(self.parse())
                self._ws()
                if s[self.i] == ",":
                    self.i += 1
                    continue
                assert s[self.i] == ")"
                self.i += 1
                break
            if op in ("+", "*"):
                acc = args[0]
                for a in args[1:]:
                    acc = self._tmp(f"{acc} {op} {a}")
                return acc
            if op in ("-", "/") and len(args) == 2:
                return self._tmp(f"{args[0]} {op} {args[1]}")
            if op == "-" and len(args) == 1:
                return self._tmp(f"-{args[0]}")
            if op == "^":
                return self._tmp(_pow(args[0], args[1]))
            if op in ("sqrt", "exp", "log"):
                return self._tmp(f"{op}({args[0]})")
            raise ValueError(f"operator {op!r}")
        m = re.compile(r"ˍ₋arg1\[(\d+)\]").match(s, self.i)
        if m:
            self.i = m.end()
            return f"x[{int(m.group(1)) - 1}]"
        m = re.compile(_num).match(s, self.i)
        if m:
            self.i = m.end()
            return repr(float(m.group(0)))
        raise ValueError("unexpected input at: " + s[self.i:self.i + 40])


def translate_sym_component(path: str) -> tuple[list[str], str]:
    text = open(path, encoding="utf-8").read()
    body = text[text.index("begin") + len("begin"):]
    body = body[:body.rindex("end")]
    body = body[:body.rindex("end")].strip()
    body = body.replace("0.333333333333", EXACT_THIRD)
    p = _Prefix(body)
    res = p.parse()
    return p.out, res


def translate_all(gen_dir: str, out_c: str) -> None:
    parts = ["/* Generated by oracle/translate_sw_ref.py from the reference checkout; not committed. */",
             "#include <math.h>", ""]
    for b in SW3:
        parts.append(translate_fd(os.path.join(gen_dir, "SW", f"H3_exec_{b}.jl"), f"ref_H3_exec_{b}"))
    for b in SW2:
        parts.append(translate_fd(os.path.join(gen_dir, "SW", f"H2_exec_{b}.jl"), f"ref_H2_exec_{b}"))
    # runtime-Symbolics iik block, one function per component, then the block
    comps = []
    for a in range(1, 4):
        for b in range(1, 4):
            for c in range(1, 4):
                body, res = translate_sym_component(
                    os.path.join(gen_dir, "SW_sym_iik", f"H3_exec_iik_{a}{b}{c}.jl"))
                name = f"ref_iik_{a}{b}{c}"
                parts.append(f"static double {name}(const double* x) {{\n" + "\n".join(body) +
                             f"\n    return {res};\n}}\n")
                comps.append(((a - 1) + 3 * (b - 1) + 9 * (c - 1), name))
    parts.append("void ref_H3_exec_iik(const double* x, double* out) {\n" +
                 "\n".join(f"    out[{f}] = {n}(x);" for f, n in comps) + "\n}\n")
    # LJ pair blocks of the AutoDiffCalculator (σ = 3.4 Å, ϵ = 0.24037 kcal/mol
    # baked in): second_order_AD.jl:25, third_order_AD.jl:26
    parts.append(translate_fd(os.path.join(gen_dir, "LJ", "H2_exec_LJ.jl"), "ref_H2_exec_LJ"))
    parts.append(translate_fd(os.path.join(gen_dir, "LJ", "H3_exec_LJ.jl"), "ref_H3_exec_LJ"))
    os.makedirs(os.path.dirname(out_c), exist_ok=True)
    with open(out_c, "w") as f:
        f.write("\n".join(parts))

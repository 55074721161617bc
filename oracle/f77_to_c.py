#!/usr/bin/env python3
"""Mechanical translation of a small Fortran 77 subset into C.

Test infrastructure: this recipe lets the oracle's hand restatements of the
reference's Fortran kernels (roeflux7.f, boundflux5.f, roejac6.f) be checked
against the reference's own source when no Fortran compiler is available.
It reads the .f files from the AERO-F tree and writes C into oracle/_ref/
(never into the repository); nothing of the product links or runs it.

Supported: fixed-form source (comment lines starting with c/C/*/!,
continuation marks in column 6), SUBROUTINE headers, IMPLICIT NONE,
REAL*8 / INTEGER declarations with explicit-shape or assumed-size (*)
arrays, assignments, IF (...) THEN / ELSE IF (...) THEN / ELSE / END IF,
DO with or without a label (label CONTINUE), END DO, RETURN, END.
Expressions follow Fortran precedence and associativity (** right
associative and above unary minus; unary minus below * and /; left to
right otherwise) and are emitted fully parenthesised, so the C compiler
evaluates them in the same order.  Literal kinds are kept: a real literal
without a D exponent is single precision, as in Fortran (emitted as a float
constant converted to double); x**n with a small integer n is repeated
multiplication, as gfortran expands it.  Intrinsics: SQRT/DSQRT, ABS/DABS,
MAX/DMAX1/MIN/DMIN1 (two or more arguments), SIGN/DSIGN.  Array indices
are 1-based, arrays column-major.  Scalar dummy arguments are passed by
pointer (Fortran calling convention); the generated function is
`<name>_f77_(...)` with every argument a pointer.

    python oracle/f77_to_c.py OUT.c file1.f [file2.f ...]
"""
from __future__ import annotations

import re
import sys

# ------------------------------------------------------------- source lines


def logical_lines(text: str) -> list[tuple[str | None, str]]:
    """Fixed-form source -> [(label, statement)] with continuations joined."""
    out: list[list] = []
    for raw in text.splitlines():
        if not raw.strip():
            continue
        if raw[0] in "cC*!":
            continue
        line = raw.rstrip("\n").expandtabs(6)
        # an inline '!' comment (not inside quotes: none in this subset)
        if "!" in line[6:]:
            line = line[:6] + line[6:].split("!", 1)[0]
        if len(line) > 5 and line[5] not in " 0" and out:
            out[-1][1] += " " + line[6:72].strip()
            continue
        label = line[:5].strip() or None
        out.append([label, line[6:72].strip()])
    return [(a, b) for a, b in out if b]


# ---------------------------------------------------------------- tokenizer
TOK = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([eEdD][+-]?\d+)?)
  | (?P<op>\*\*|\.(?:gt|ge|lt|le|eq|ne|and|or|not)\.|[-+*/(),=])
  | (?P<id>[A-Za-z_][A-Za-z_0-9]*)
  | (?P<ws>\s+)
""", re.X | re.I)


def tokens(s: str) -> list[tuple[str, str]]:
    out, pos = [], 0
    while pos < len(s):
        m = TOK.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot tokenise at {s[pos:]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        v = m.group(kind)
        if kind == "op":
            v = v.lower()
        if kind == "id":
            v = v.lower()
        out.append((kind, v))
    return out


# ------------------------------------------------------------- expressions
class Parser:
    """Recursive descent over Fortran precedence, emitting parenthesised C."""

    def __init__(self, toks, tr):
        self.t, self.i, self.tr = toks, 0, tr

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, v=None):
        tok = self.peek()
        if v is not None and tok[1] != v:
            raise SyntaxError(f"expected {v!r}, got {tok!r}")
        self.i += 1
        return tok

    # or > and > not > relational > additive > multiplicative > unary > power
    def expr(self):
        a = self.and_()
        while self.peek()[1] == ".or.":
            self.take()
            a = f"({a} || {self.and_()})"
        return a

    def and_(self):
        a = self.not_()
        while self.peek()[1] == ".and.":
            self.take()
            a = f"({a} && {self.not_()})"
        return a

    def not_(self):
        if self.peek()[1] == ".not.":
            self.take()
            return f"(!{self.not_()})"
        return self.rel()

    REL = {".gt.": ">", ".ge.": ">=", ".lt.": "<", ".le.": "<=", ".eq.": "==", ".ne.": "!="}

    def rel(self):
        a = self.add()
        if self.peek()[1] in self.REL:
            op = self.REL[self.take()[1]]
            b = self.add()
            return f"({a} {op} {b})"
        return a

    def add(self):
        # a leading sign applies to the first term (lower precedence than *)
        if self.peek()[1] in ("+", "-"):
            sgn = self.take()[1]
            a = self.mul()
            a = f"(-{a})" if sgn == "-" else a
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            b = self.mul()
            a = f"({a} {op} {b})"
        return a

    def mul(self):
        a = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            b = self.power()
            a = f"({a} {op} {b})"
        return a

    def power(self):
        base = self.primary()
        if self.peek()[1] == "**":
            self.take()
            # right associative; the exponent may carry a sign
            if self.peek()[1] in ("+", "-"):
                sgn = self.take()[1]
                e = self.power()
                e = f"(-{e})" if sgn == "-" else e
            else:
                e = self.power()
            m = re.fullmatch(r"\(?(\d+)\)?", e)
            if m and 1 <= int(m.group(1)) <= 4:
                n = int(m.group(1))
                if n == 1:
                    return base
                # gfortran expands small integer powers by multiplication:
                # x**2 = x*x, x**3 = x*x*x, x**4 = (x*x)*(x*x)
                if n == 2:
                    return f"({base} * {base})"
                if n == 3:
                    return f"(({base} * {base}) * {base})"
                return f"(({base} * {base}) * ({base} * {base}))"
            return f"pow({base}, {e})"
        return base

    def primary(self):
        kind, v = self.take()
        if kind == "num":
            return self.tr.literal(v)
        if v == "(":
            e = self.expr()
            self.take(")")
            return f"({e})"
        if kind == "id":
            if self.peek()[1] == "(":
                self.take("(")
                args = [self.expr()]
                while self.peek()[1] == ",":
                    self.take()
                    args.append(self.expr())
                self.take(")")
                return self.tr.call_or_index(v, args)
            return self.tr.scalar(v)
        raise SyntaxError(f"unexpected token {v!r}")


# --------------------------------------------------------------- translator
INTRINSIC = {"sqrt": "sqrt", "dsqrt": "sqrt", "abs": "fabs", "dabs": "fabs"}


class Unit:
    def __init__(self, name, args):
        self.name, self.args = name, args
        self.types: dict[str, str] = {}
        self.dims: dict[str, list[str]] = {}
        self.body: list[str] = []
        self.depth = 1
        self.do_labels: list[str] = []

    # names
    def literal(self, v: str) -> str:
        if re.fullmatch(r"\d+", v):
            return v
        if re.search(r"[dD]", v):
            return "(" + v.lower().replace("d", "e") + ")"
        mant = v if re.search(r"[eE]", v) else (v + "e0" if "." in v else v)
        return f"((double){mant}f)"

    def scalar(self, v: str) -> str:
        if v in self.dims:
            raise SyntaxError(f"array {v} used without index")
        return f"(*{v})" if v in self.args else v

    def call_or_index(self, v: str, args: list[str]) -> str:
        if v in self.dims:
            dims = self.dims[v]
            if len(args) == 1:
                return f"{v}[({args[0]}) - 1]"
            if len(args) == 2:
                return f"{v}[(({args[0]}) - 1) + (({args[1]}) - 1) * ({dims[0]})]"
            raise SyntaxError(f"rank-{len(args)} array {v}")
        if v in INTRINSIC:
            return f"{INTRINSIC[v]}({args[0]})"
        if v in ("max", "dmax1", "amax1", "min", "dmin1", "amin1"):
            fn = "f77_max" if "max" in v else "f77_min"
            acc = args[0]
            for a in args[1:]:
                acc = f"{fn}({acc}, {a})"
            return acc
        if v in ("sign", "dsign"):
            return f"f77_sign({args[0]}, {args[1]})"
        raise SyntaxError(f"unknown function or array {v}")

    def emit(self, s: str):
        self.body.append("  " * self.depth + s)

    def expr(self, s: str) -> str:
        p = Parser(tokens(s), self)
        e = p.expr()
        if p.i != len(p.t):
            raise SyntaxError(f"trailing tokens in {s!r}")
        return e

    def lvalue(self, s: str) -> str:
        return self.expr(s)

    def declare(self, typ: str, rest: str):
        # split at top-level commas
        items, depth, cur = [], 0, ""
        for ch in rest:
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
            if ch == "," and depth == 0:
                items.append(cur)
                cur = ""
            else:
                cur += ch
        items.append(cur)
        for it in items:
            it = it.strip().lower()
            if not it:
                continue
            m = re.fullmatch(r"([a-z_][a-z_0-9]*)\s*(\((.*)\))?", it)
            if not m:
                raise SyntaxError(f"declaration {it!r}")
            name = m.group(1)
            self.types[name] = typ
            if m.group(2):
                self.dims[name] = [d.strip() for d in m.group(3).split(",")]

    def statement(self, label: str | None, st: str):
        low = st.lower()
        if label and label in self.do_labels and re.fullmatch(r"continue", low):
            self.depth -= 1
            self.emit("}")
            self.do_labels.remove(label)
            return
        if label and not re.fullmatch(r"continue", low):
            raise SyntaxError(f"labelled statement {st!r}")
        if low == "continue":
            return
        if low.startswith("implicit none"):
            return
        m = re.fullmatch(r"(real\*8|integer|double precision)\s+(.*)", st, re.I)
        if m:
            self.declare("int" if m.group(1).lower() == "integer" else "double", m.group(2))
            return
        m = re.fullmatch(r"if\s*\((.*)\)\s*then", st, re.I)
        if m:
            self.emit(f"if ({self.expr(m.group(1))}) {{")
            self.depth += 1
            return
        m = re.fullmatch(r"else\s*if\s*\((.*)\)\s*then", st, re.I)
        if m:
            self.depth -= 1
            self.emit(f"}} else if ({self.expr(m.group(1))}) {{")
            self.depth += 1
            return
        if re.fullmatch(r"else", low):
            self.depth -= 1
            self.emit("} else {")
            self.depth += 1
            return
        if re.fullmatch(r"end\s*if", low) or re.fullmatch(r"end\s*do", low):
            self.depth -= 1
            self.emit("}")
            return
        m = re.fullmatch(r"do\s+(\d+\s+)?([a-z_][a-z_0-9]*)\s*=\s*(.*)", st, re.I)
        if m:
            lab, var = m.group(1), m.group(2).lower()
            parts = [p.strip() for p in m.group(3).split(",")]
            if len(parts) != 2:
                raise SyntaxError(f"DO with a step: {st!r}")
            lo, hi = self.expr(parts[0]), self.expr(parts[1])
            self.emit(f"for ({var} = {lo}; {var} <= {hi}; ++{var}) {{")
            self.depth += 1
            if lab:
                self.do_labels.append(lab.strip())
            return
        if low == "return":
            self.emit("return;")
            return
        m = re.fullmatch(r"([a-z_][a-z_0-9]*\s*(\(.*?\))?)\s*=\s*(.*)", st, re.I)
        if m:
            self.emit(f"{self.lvalue(m.group(1))} = {self.expr(m.group(3))};")
            return
        raise SyntaxError(f"unsupported statement {st!r}")

    def c_source(self) -> str:
        params = []
        for a in self.args:
            t = self.types.get(a)
            if t is None:
                raise SyntaxError(f"argument {a} has no declared type")
            params.append(f"{t}* {a}")
        lines = [f"void {self.name}_f77_({', '.join(params)}) {{"]
        for v, t in self.types.items():
            if v in self.args:
                continue
            if v in self.dims:
                size = 1
                for d in self.dims[v]:
                    size *= int(d)
                lines.append(f"  {t} {v}[{size}];")
            else:
                lines.append(f"  {t} {v};")
        lines += self.body
        lines.append("}")
        return "\n".join(lines)


def translate(text: str) -> list[str]:
    units, cur = [], None
    for label, st in logical_lines(text):
        low = st.lower()
        m = re.fullmatch(r"subroutine\s+([a-z_0-9]+)\s*\((.*)\)", st, re.I)
        if m:
            cur = Unit(m.group(1).lower(), [a.strip().lower() for a in m.group(2).split(",")])
            continue
        if re.fullmatch(r"end", low):
            units.append(cur.c_source())
            cur = None
            continue
        if cur is None:
            raise SyntaxError(f"statement outside a subroutine: {st!r}")
        cur.statement(label, st)
    return units


PRELUDE = """/* Generated by oracle/f77_to_c.py from the reference's Fortran sources;
 * test infrastructure, not part of the repository. */
#include <math.h>
static double f77_max(double a, double b) { return a > b ? a : b; }
static double f77_min(double a, double b) { return a < b ? a : b; }
static double f77_sign(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }
"""


def main(argv):
    out, srcs = argv[1], argv[2:]
    parts = [PRELUDE]
    for s in srcs:
        with open(s) as f:
            parts += translate(f.read())
    with open(out, "w") as f:
        f.write("\n\n".join(parts) + "\n")


if __name__ == "__main__":
    main(sys.argv)

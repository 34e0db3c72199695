"""Mechanism table generator: parses a FlameMaster-generated Fortran mechanism file
(the ``*F.f90`` + ``*F90.h`` pair the finite-rate chemistry path links as a plugin) into a
data table.

The reference links exactly one mechanism as a set of external Fortran symbols
(``PRODRATES``, ``GETLINDRATECOEFF``, ``COMPTHERMODATA``, ``GETMOLARMASS`` …; template in
combustion/mechanism.f90:17-108). Here a mechanism is data instead: this module reads the
straight-line Fortran statement by statement and records

* third-body sums ``M(j) = sum_k eff_jk C(k)`` in statement order
  (e.g. combustion/grimech30F.f90:33-606);
* every rate-constant slot ``K(r)``: modified Arrhenius ``A*exp(n*LT +- E/RT)``, a bare ``A``,
  or a Troe/Lindemann falloff call ``GETLINDRATECOEFF(TEMP,PRESSURE,K0TROE,KINFTROE,FCTROE,M(j))``
  with its k0/kinf/Fc expressions (grimech30F.f90:608-1604, HYDROGENF.f90:59-161);
* reaction rates ``W(r) = K(r)*C(a)*C(b)...[*M(j)]`` (grimech30F.f90:1605-2028);
* production rates ``CDOT(k) = +-nu*W(r) ...`` as ordered signed term lists
  (grimech30F.f90:2029-2579);
* NASA-7 enthalpy/heat-capacity Horner polynomials for both ranges, split at ``T.GT.1000``
  (COMPTHERMODATA, grimech30F.f90:2925-3516);
* molar masses, species names, mu coefficients and k/eps (getters, HYDROGENF.f90:366-496).

Every numeric literal keeps its source text. Its kind follows Fortran rules for the
reference's build (Makefile.in:23-24 has no default-real promotion flag): a ``D`` exponent or
a ``_DP`` suffix is double precision, a plain real literal is *default real* (float32, then
widened), an integer literal is exact. :func:`literal_value` applies that rule.

The ``.h`` DATA arrays (HYDROGENF90.h:45-127) are not used: PRODRATES never reads them and
their falloff pre-exponentials are in other units.

Run ``python -m tiger_nga_b200.mechgen <reference combustion dir> <out dir>`` to regenerate the
committed tables under ``tiger_nga_b200/mechanisms/``.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import struct
import sys
from dataclasses import dataclass
from typing import Any

# --------------------------------------------------------------------------------------
# literals
# --------------------------------------------------------------------------------------


def literal_kind(text: str) -> str:
    """Fortran kind of a numeric literal as written in the mechanism source.

    ``'f64'`` for a D exponent or ``_DP`` suffix, ``'f32'`` for a default-real literal,
    ``'int'`` for an integer literal.
    """
    t = text.strip()
    if t.upper().endswith("_DP"):
        return "f64"
    if "d" in t.lower():
        return "f64"
    if "." in t or "e" in t.lower():
        return "f32"
    return "int"


def _f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", x))[0]


def literal_value(text: str, mode: str = "f32") -> float:
    """Value of a literal as the reference binary sees it.

    ``mode='f32'`` (default) rounds default-real literals to float32 like the reference build;
    ``mode='f64'`` reads every literal as a double (what ``-fdefault-real-8`` would do).
    """
    t = text.strip()
    kind = literal_kind(t)
    s = t
    if s.upper().endswith("_DP"):
        s = s[:-3]
    s = s.replace("D", "E").replace("d", "e")
    v = float(s)
    if kind == "f32" and mode == "f32":
        return _f32(v)
    return v


# --------------------------------------------------------------------------------------
# statements and expressions
# --------------------------------------------------------------------------------------


def read_statements(path: str) -> list[tuple[int, str]]:
    """Fortran free-form statements with ``&`` continuations joined and comments dropped.

    Returns ``(first source line, text)`` pairs.
    """
    out: list[tuple[int, str]] = []
    cur = ""
    start = 0
    with open(path, "r", errors="replace") as fh:
        for lineno, raw in enumerate(fh, 1):
            line = raw.rstrip("\n")
            # strip comments outside string literals
            buf = []
            q = None
            for ch in line:
                if q:
                    buf.append(ch)
                    if ch == q:
                        q = None
                    continue
                if ch in "'\"":
                    q = ch
                    buf.append(ch)
                    continue
                if ch == "!":
                    break
                buf.append(ch)
            s = "".join(buf).rstrip()
            if not cur:
                start = lineno
            if s.endswith("&"):
                cur += s[:-1] + " "
                continue
            cur += s
            if cur.strip():
                out.append((start, " ".join(cur.split())))
            cur = ""
    return out


_TOKEN = re.compile(
    r"\s*(?:"
    r"(?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eEdD][+-]?\d+)?(?:_DP)?)"
    r"|(?P<name>[A-Za-z_][A-Za-z_0-9]*)"
    r"|(?P<op>\*\*|[-+*/(),=])"
    r")"
)


@dataclass
class Node:
    kind: str  # num | var | idx | call | neg | add | sub | mul | div | pow
    a: Any = None
    b: Any = None
    args: Any = None

    def __repr__(self) -> str:  # compact debug form
        if self.kind == "num":
            return self.a
        if self.kind == "var":
            return self.a
        if self.kind in ("idx", "call"):
            return f"{self.a}({','.join(map(repr, self.args))})"
        if self.kind == "neg":
            return f"(-{self.a!r})"
        op = {"add": "+", "sub": "-", "mul": "*", "div": "/", "pow": "**"}[self.kind]
        return f"({self.a!r}{op}{self.b!r})"


def tokenize(s: str) -> list[tuple[str, str]]:
    toks = []
    pos = 0
    s = s.rstrip()
    while pos < len(s):
        m = _TOKEN.match(s, pos)
        if not m or m.end() == pos:
            raise ValueError(f"cannot tokenize at {s[pos:pos + 30]!r} in {s!r}")
        for k in ("num", "name", "op"):
            if m.group(k) is not None:
                v = m.group(k)
                toks.append((k, v.upper() if k == "name" else v))
                break
        pos = m.end()
    return toks


class _Parser:
    """Recursive-descent parser with Fortran precedence: ``**`` (right assoc) binds tighter
    than ``* /``, which bind tighter than unary and binary ``+ -``."""

    ARRAYS = {"K", "W", "C", "M", "CDOT", "H", "CP", "MM", "MUCOEFF", "KOVEREPS", "NAMES"}

    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise ValueError(f"expected {val!r}, got {tok!r}")
        self.i += 1
        return tok

    def expr(self) -> Node:
        k, v = self.peek()
        if v in ("+", "-"):
            self.take()
            node = self.term()
            if v == "-":
                node = Node("neg", node)
        else:
            node = self.term()
        while self.peek()[1] in ("+", "-"):
            _, op = self.take()
            rhs = self.term()
            node = Node("add" if op == "+" else "sub", node, rhs)
        return node

    def term(self) -> Node:
        node = self.factor()
        while self.peek()[1] in ("*", "/"):
            _, op = self.take()
            rhs = self.factor()
            node = Node("mul" if op == "*" else "div", node, rhs)
        return node

    def factor(self) -> Node:
        base = self.primary()
        if self.peek()[1] == "**":
            self.take()
            return Node("pow", base, self.factor())
        return base

    def primary(self) -> Node:
        k, v = self.take()
        if k == "num":
            return Node("num", v)
        if k == "name":
            if self.peek()[1] == "(":
                self.take("(")
                args = [self.expr()]
                while self.peek()[1] == ",":
                    self.take(",")
                    args.append(self.expr())
                self.take(")")
                return Node("idx" if v in self.ARRAYS else "call", v, args=args)
            return Node("var", v)
        if v == "(":
            node = self.expr()
            self.take(")")
            return node
        raise ValueError(f"unexpected token {v!r}")


def parse_expr(s: str) -> Node:
    p = _Parser(tokenize(s))
    node = p.expr()
    if p.i != len(p.t):
        raise ValueError(f"trailing tokens in {s!r}: {p.t[p.i:]}")
    return node


def parse_assignment(s: str) -> tuple[Node, Node]:
    toks = tokenize(s)
    depth = 0
    for i, (k, v) in enumerate(toks):
        if v == "(":
            depth += 1
        elif v == ")":
            depth -= 1
        elif v == "=" and depth == 0:
            lp = _Parser(toks[:i])
            lhs = lp.primary()
            rp = _Parser(toks[i + 1:])
            rhs = rp.expr()
            if rp.i != len(rp.t) or lp.i != len(lp.t):
                raise ValueError(f"bad assignment {s!r}")
            return lhs, rhs
    raise ValueError(f"not an assignment: {s!r}")


# --------------------------------------------------------------------------------------
# header parameters
# --------------------------------------------------------------------------------------


def parse_header(path: str) -> dict[str, int]:
    """Integer PARAMETERs (species S*, slots R*, third-body sets MM*) from ``*F90.h``."""
    params: dict[str, int] = {}
    for _, st in read_statements(path):
        if not re.match(r"(?i)integer\s*,\s*parameter\s*::", st):
            continue
        body = st.split("::", 1)[1]
        for item in body.split(","):
            if "=" not in item:
                continue
            name, val = item.split("=")
            name = name.strip().upper()
            val = val.strip()
            if re.fullmatch(r"\d+", val):
                params[name] = int(val)
    return params


# --------------------------------------------------------------------------------------
# pattern matching helpers
# --------------------------------------------------------------------------------------


def _flatten_additive(node: Node) -> list[tuple[int, Node]]:
    """Left-to-right list of (sign, term) for a chain of + / - (and a leading unary minus)."""
    if node.kind == "add":
        return _flatten_additive(node.a) + [(+1, node.b)]
    if node.kind == "sub":
        return _flatten_additive(node.a) + [(-1, node.b)]
    if node.kind == "neg":
        return [(-1, node.a)]
    return [(+1, node)]


def _flatten_product(node: Node) -> list[Node]:
    if node.kind == "mul":
        return _flatten_product(node.a) + [node.b]
    return [node]


def _num(node: Node) -> str:
    if node.kind != "num":
        raise ValueError(f"expected literal, got {node!r}")
    return node.a


def _signed(sign: int, text: str) -> str:
    return text if sign > 0 else "-" + text


def _idx_name(node: Node, arr: str, params: dict[str, int]) -> int:
    if node.kind != "idx" or node.a != arr or len(node.args) != 1 or node.args[0].kind != "var":
        raise ValueError(f"expected {arr}(name), got {node!r}")
    return params[node.args[0].a]


def _arrhenius(node: Node) -> dict:
    """``A`` or ``A*exp(arg)`` with arg = [+-] n*LT [+- E/RT] | [+-] E/RT.

    Signs are folded into the literal text: IEEE negation is exact, so
    ``-(n*LT) - E/RT`` equals ``(-n)*LT + (-E)/RT`` bit for bit.
    """
    if node.kind == "num":
        return {"A": node.a, "n": None, "E": None}
    if node.kind != "mul" or node.a.kind != "num" or node.b.kind != "call" or node.b.a != "EXP":
        raise ValueError(f"not an Arrhenius form: {node!r}")
    A = node.a.a
    n = E = None
    terms = _flatten_additive(node.b.args[0])
    if len(terms) > 2:
        raise ValueError(f"unexpected exponent {node!r}")
    for pos, (sign, t) in enumerate(terms):
        if t.kind == "mul" and t.b.kind == "var" and t.b.a == "LT" and pos == 0:
            n = _signed(sign, _num(t.a))
        elif t.kind == "div" and t.b.kind == "var" and t.b.a == "RT":
            E = _signed(sign, _num(t.a))
        else:
            raise ValueError(f"unexpected exponent term {t!r}")
    return {"A": A, "n": n, "E": E}


def _fcent(node: Node) -> list[dict]:
    """Troe F_cent = sum of ``a*EXP(-TEMP/T3)`` / ``a*EXP(-T2/TEMP)`` terms, in order."""
    terms = []
    for sign, t in _flatten_additive(node):
        if sign != +1 or t.kind != "mul" or t.a.kind != "num" or t.b.kind != "call" or t.b.a != "EXP":
            raise ValueError(f"unexpected Fc term {t!r}")
        arg = t.b.args[0]
        if arg.kind != "neg":
            raise ValueError(f"unexpected Fc exponent {arg!r}")
        inner = arg.a
        if inner.kind != "div":
            raise ValueError(f"unexpected Fc exponent {arg!r}")
        if inner.a.kind == "var" and inner.a.a == "TEMP":
            terms.append({"a": t.a.a, "form": "T_over", "x": _num(inner.b)})
        elif inner.b.kind == "var" and inner.b.a == "TEMP":
            terms.append({"a": t.a.a, "form": "over_T", "x": _num(inner.a)})
        else:
            raise ValueError(f"unexpected Fc exponent {arg!r}")
    return terms


def _horner(node: Node) -> list[str]:
    """Coefficients of ``a1 + T*(a2 + T*(... + T*(aK)))`` (innermost may be a lone literal)."""
    coefs = []
    cur = node
    while True:
        if cur.kind == "num":
            coefs.append(cur.a)
            return coefs
        if cur.kind == "neg" and cur.a.kind == "num":
            coefs.append("-" + cur.a.a)
            return coefs
        if cur.kind in ("add", "sub"):
            lhs, rhs = cur.a, cur.b
            if lhs.kind == "neg" and lhs.a.kind == "num":
                coefs.append("-" + lhs.a.a)
            elif lhs.kind == "num":
                coefs.append(lhs.a)
            else:
                raise ValueError(f"bad Horner head {lhs!r}")
            if rhs.kind != "mul" or rhs.a.kind != "var" or rhs.a.a != "T":
                raise ValueError(f"bad Horner tail {rhs!r}")
            if cur.kind == "sub":
                raise ValueError("subtracted Horner tail not supported")
            cur = rhs.b
            continue
        raise ValueError(f"bad Horner node {cur!r}")


def _thermo_h(rhs: Node) -> dict:
    # c0 * ( T * (horner) +- a6 )
    if rhs.kind != "mul" or rhs.a.kind != "num":
        raise ValueError(f"bad H statement {rhs!r}")
    inner = rhs.b
    if inner.kind not in ("add", "sub") or inner.a.kind != "mul" or inner.a.a.kind != "var" or inner.a.a.a != "T":
        raise ValueError(f"bad H body {inner!r}")
    a6 = _num(inner.b)
    return {"c0": rhs.a.a, "a": _horner(inner.a.b), "a6": a6 if inner.kind == "add" else "-" + a6}


def _thermo_cp(rhs: Node) -> dict:
    if rhs.kind != "mul" or rhs.a.kind != "num":
        raise ValueError(f"bad CP statement {rhs!r}")
    return {"c0": rhs.a.a, "b": _horner(rhs.b)}


# --------------------------------------------------------------------------------------
# routine extraction
# --------------------------------------------------------------------------------------


def _routine(stmts, name: str) -> list[tuple[int, str]]:
    """Statements strictly inside SUBROUTINE/FUNCTION ``name`` (header and END excluded)."""
    start = None
    for i, (_, s) in enumerate(stmts):
        u = s.upper()
        if start is None:
            if re.match(rf"(DOUBLE PRECISION\s+FUNCTION|SUBROUTINE)\s+{name}\s*\(", u):
                start = i + 1
        elif u == "END":
            return stmts[start:i]
    raise ValueError(f"routine {name} not found")


_SKIP = re.compile(r"(?i)^(implicit|include|real|integer|double precision|character|parameter)\b")


def parse_mechanism(f90: str, h: str, name: str) -> dict:
    """Parse one generated mechanism into the table dict stored as JSON."""
    params = parse_header(h)
    stmts = read_statements(f90)
    nspec = params["SEND"] - 1
    nslot = params["REND"] - 1
    nmset = params["MEND"] - 1
    sp_names = sorted((v, k) for k, v in params.items() if k.startswith("S") and k != "SEND" and v <= nspec)
    slot_names = {v: k for k, v in params.items() if re.fullmatch(r"R\d+[FB]?", k)}
    lineof: dict[str, int] = {}

    third_body: list[list[list]] = [[] for _ in range(nmset)]
    kslots: list[dict | None] = [None] * nslot
    wslots: list[dict | None] = [None] * nslot
    cdot: list[list[list] | None] = [None] * nspec
    state = {"K0TROE": None, "KINFTROE": None, "FCTROE": None}
    k0_consumed = True

    for lineno, st in _routine(stmts, "PRODRATES"):
        if _SKIP.match(st):
            continue
        lhs, rhs = parse_assignment(st)
        if lhs.kind == "var" and lhs.a in ("LT", "RT"):
            want = {"LT": "DLOG(TEMP)", "RT": "(RGAS*TEMP)"}[lhs.a]
            if repr(rhs).replace(" ", "") != want:
                raise ValueError(f"{lhs.a} statement changed: {st}")
            continue
        if lhs.kind == "var" and lhs.a in state:
            if lhs.a == "FCTROE":
                state["FCTROE"] = _fcent(rhs)
            else:
                state[lhs.a] = _arrhenius(rhs)
                if lhs.a == "K0TROE":
                    k0_consumed = False
            continue
        if lhs.kind != "idx":
            raise ValueError(f"unhandled statement at line {lineno}: {st}")
        arr = lhs.a
        if arr == "M":
            j = _idx_name(lhs, "M", params) - 1
            terms = _flatten_additive(rhs)
            out = third_body[j]
            for pos, (sign, t) in enumerate(terms):
                if sign != +1:
                    raise ValueError(f"negative third-body term at {lineno}")
                if t.kind == "idx" and t.a == "M":
                    if pos != 0 or _idx_name(t, "M", params) - 1 != j or not out:
                        raise ValueError(f"bad M continuation at {lineno}")
                    continue
                if t.kind == "idx" and t.a == "C":
                    out.append([_idx_name(t, "C", params) - 1, "1"])
                elif t.kind == "mul" and t.a.kind == "num" and t.b.kind == "idx" and t.b.a == "C":
                    out.append([_idx_name(t.b, "C", params) - 1, t.a.a])
                else:
                    raise ValueError(f"bad third-body term {t!r} at {lineno}")
        elif arr == "K":
            r = _idx_name(lhs, "K", params) - 1
            if kslots[r] is not None:
                raise ValueError(f"slot assigned twice at {lineno}")
            lineof[f"K{r}"] = lineno
            if rhs.kind == "call" and rhs.a == "GETLINDRATECOEFF":
                args = [repr(a) for a in rhs.args]
                if args[:5] != ["TEMP", "PRESSURE", "K0TROE", "KINFTROE", "FCTROE"]:
                    raise ValueError(f"unexpected falloff call at {lineno}: {args}")
                if k0_consumed:
                    raise ValueError(f"falloff at {lineno} reuses a K0TROE already modified in place")
                if None in state.values():
                    raise ValueError(f"falloff at {lineno} before k0/kinf/Fc were set")
                mj = _idx_name(rhs.args[5], "M", params) - 1
                kslots[r] = {"type": "falloff", "k0": dict(state["K0TROE"]), "kinf": dict(state["KINFTROE"]),
                             "fc": [dict(t) for t in state["FCTROE"]], "M": mj, "line": lineno}
                k0_consumed = True  # GETLINDRATECOEFF overwrites its K0 argument
            else:
                d = _arrhenius(rhs)
                d.update({"type": "arrhenius", "line": lineno})
                kslots[r] = d
        elif arr == "W":
            r = _idx_name(lhs, "W", params) - 1
            factors = _flatten_product(rhs)
            if _idx_name(factors[0], "K", params) - 1 != r:
                raise ValueError(f"W({r}) does not use its own K at {lineno}")
            species, mj = [], -1
            for f in factors[1:]:
                if f.kind == "idx" and f.a == "C" and mj < 0:
                    species.append(_idx_name(f, "C", params) - 1)
                elif f.kind == "idx" and f.a == "M" and mj < 0:
                    mj = _idx_name(f, "M", params) - 1
                else:
                    raise ValueError(f"bad rate factor {f!r} at {lineno}")
            wslots[r] = {"C": species, "M": mj, "line": lineno}
        elif arr == "CDOT":
            k = _idx_name(lhs, "CDOT", params) - 1
            if rhs.kind == "num":
                if literal_value(rhs.a) != 0.0:
                    raise ValueError(f"nonzero constant CDOT at {lineno}")
                cdot[k] = []
                continue
            terms = _flatten_additive(rhs)
            cont = terms[0][1].kind == "idx" and terms[0][1].a == "CDOT"
            if cont:
                if _idx_name(terms[0][1], "CDOT", params) - 1 != k or cdot[k] is None or terms[0][0] != 1:
                    raise ValueError(f"bad CDOT continuation at {lineno}")
                terms = terms[1:]
                out = cdot[k]
            else:
                if cdot[k] is not None:
                    raise ValueError(f"CDOT assigned twice at {lineno}")
                out = cdot[k] = []
            for sign, t in terms:
                if t.kind == "idx" and t.a == "W":
                    out.append([sign, "1", _idx_name(t, "W", params) - 1])
                elif t.kind == "mul" and t.a.kind == "num" and t.b.kind == "idx" and t.b.a == "W":
                    out.append([sign, t.a.a, _idx_name(t.b, "W", params) - 1])
                else:
                    raise ValueError(f"bad CDOT term {t!r} at {lineno}")
        else:
            raise ValueError(f"unhandled array {arr} at {lineno}: {st}")

    missing = [i for i in range(nslot) if kslots[i] is None or wslots[i] is None]
    if missing:
        raise ValueError(f"slots without K or W: {missing[:10]}")
    if any(c is None for c in cdot):
        raise ValueError("species without CDOT")

    # ---- GETLINDRATECOEFF: check it is the Troe form the table encodes
    lind = [s for _, s in _routine(stmts, "GETLINDRATECOEFF")]
    lind_text = " ".join(lind).upper().replace(" ", "")
    for frag in ("ITROE=1", "NTMP=0.75-1.27*DLOG10(FC)", "CCOEFF=-0.4-0.67*DLOG10(FC)", "DCOEFF=0.14",
                 "K0=K0*CONC/MAX(KINF,1.0D-60)", "F=FC**(1.0/(F*F+1.0))",
                 "GETLINDRATECOEFF=KINF*F*K0/(1.0+K0)", "CONC=PRESSURE/(R*TEMP)", "PARAMETER(R=8314.34)"):
        if frag not in lind_text:
            raise ValueError(f"GETLINDRATECOEFF differs from the Troe form: missing {frag}")

    # ---- thermo
    thermo = {"hi": [None] * nspec, "lo": [None] * nspec}
    body = _routine(stmts, "COMPTHERMODATA")
    rng = None
    tmid = None
    for lineno, st in body:
        u = st.upper().replace(" ", "")
        if _SKIP.match(st):
            continue
        m = re.fullmatch(r"IF\(T\.GT\.([0-9.]+(?:_DP)?)\)THEN", u)
        if m:
            tmid = m.group(1)
            rng = "hi"
            continue
        if u == "ELSE":
            rng = "lo"
            continue
        if u in ("ENDIF", "END IF"):
            rng = None
            continue
        lhs, rhs = parse_assignment(st)
        k = _idx_name(lhs, lhs.a, params) - 1
        ent = thermo[rng][k] or {}
        if lhs.a == "H":
            ent.update(_thermo_h(rhs))
        elif lhs.a == "CP":
            c = _thermo_cp(rhs)
            if "c0" in ent and ent["c0"] != c["c0"]:
                raise ValueError("H and CP use different R/W factors")
            ent.update(c)
        else:
            raise ValueError(f"unexpected thermo statement {st}")
        thermo[rng][k] = ent
    for r in ("hi", "lo"):
        for k, ent in enumerate(thermo[r]):
            if not ent or len(ent.get("a", [])) != 5 or len(ent.get("b", [])) != 5:
                raise ValueError(f"incomplete thermo for species {k} ({r})")

    def getter(rname: str, arr: str) -> list[str]:
        vals = [None] * nspec
        for _, st in _routine(stmts, rname):
            if _SKIP.match(st):
                continue
            lhs, rhs = parse_assignment(st)
            vals[_idx_name(lhs, arr, params) - 1] = _num(rhs) if rhs.kind == "num" else "-" + _num(rhs.a)
        return vals

    names = [None] * nspec
    for _, st in _routine(stmts, "GETSPECIESNAMES"):
        m = re.match(r"(?i)NAMES\((\w+)\)\s*=\s*'([^']*)'", st)
        if m:
            names[params[m.group(1).upper()] - 1] = m.group(2).strip()

    nreac = None
    for _, st in _routine(stmts, "GETNREACTIONS"):
        m = re.match(r"(?i)NREACTIONS\s*=\s*(\d+)", st)
        if m:
            nreac = int(m.group(1))
    if nreac != nslot:
        raise ValueError(f"GETNREACTIONS {nreac} != slot count {nslot}")

    with open(f90, "rb") as fh:
        f90_sha = hashlib.sha256(fh.read()).hexdigest()
    with open(h, "rb") as fh:
        h_sha = hashlib.sha256(fh.read()).hexdigest()

    return {
        "format": "tiger-chem-mechanism/1",
        "name": name,
        "provenance": {
            "source": "combustion/" + os.path.basename(f90),
            "header": "combustion/" + os.path.basename(h),
            "sha256": f90_sha,
            "header_sha256": h_sha,
            "generator": "tiger_nga_b200.mechgen",
        },
        "rgas": "8314.34",
        "n_species": nspec,
        "n_slots": nslot,
        "n_thirdbody": nmset,
        "species": names,
        "species_params": [n for _, n in sp_names],
        "slot_names": [slot_names[i + 1] for i in range(nslot)],
        "molar_mass": getter("GETMOLARMASS", "MM"),
        "mucoeff": getter("GETMUCOEFF", "MUCOEFF"),
        "koveps": getter("GETKOVEREPS", "KOVEREPS"),
        "third_body": third_body,
        "k": kslots,
        "w": wslots,
        "cdot": cdot,
        "thermo": {"tmid": tmid, "hi": thermo["hi"], "lo": thermo["lo"]},
    }


BUILTIN = {
    "hydrogen": ("HYDROGENF.f90", "HYDROGENF90.h"),
    "grimech30": ("grimech30F.f90", "grimech30F90.h"),
    "dme39": ("DME39F.f90", "DME39F90.h"),
}


def main(argv: list[str]) -> int:
    if len(argv) != 3:
        print("usage: python -m tiger_nga_b200.mechgen <combustion dir> <out dir>", file=sys.stderr)
        return 2
    src, out = argv[1], argv[2]
    os.makedirs(out, exist_ok=True)
    for name, (f90, h) in BUILTIN.items():
        tab = parse_mechanism(os.path.join(src, f90), os.path.join(src, h), name)
        path = os.path.join(out, name + ".json")
        with open(path, "w") as fh:
            json.dump(tab, fh, indent=0, separators=(",", ":"))
            fh.write("\n")
        print(f"{name}: {tab['n_species']} species, {tab['n_slots']} slots, "
              f"{sum(1 for k in tab['k'] if k['type'] == 'falloff')} falloff, "
              f"{tab['n_thirdbody']} third-body sets -> {path}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))

"""Constraint expressions: C integer expressions -> postfix programs.

The reference pastes each constraint string into generated CUDA as a C
expression (system/tmine/Query.py:186-190 renders `auto f = nodeFeature[id];
return <cond>;`, Query.py:242-247 the same for edges, and Query.py:90-98
rewrites `e<i>` in a filter to `edgeFeature[eid<i>]`; KernelGen.py:530-534
wraps it around the count).  Here the string is parsed with C's grammar and
typing rules for the integer subset (int and long operands; unsigned
literals are rejected) and compiled to the program format of
include/everest_b200.h, which one precompiled kernel interprets.

`f` is the feature (an int); `e<i>` is the feature of the edge matched to
motif edge i.  `evaluate` is a host interpreter of the same program format,
used by tests and to check programs.
"""
from __future__ import annotations

import re
from typing import List, Optional, Sequence, Tuple

OP = dict(CONST=1, VAR=2, NEG=3, NOT=4, BNOT=5, ADD=6, SUB=7, MUL=8, DIV=9, MOD=10, SHL=11, SHR=12,
          LT=13, LE=14, GT=15, GE=16, EQ=17, NE=18, BAND=19, BXOR=20, BOR=21, LAND=22, LOR=23, COND=24)
WRAP32 = 0x80
PROG_MAX = 48
PROG_STACK = 16
INT_MIN, INT_MAX = -(1 << 31), (1 << 31) - 1
LONG_MIN, LONG_MAX = -(1 << 63), (1 << 63) - 1

_BINARY = {
    "||": (2, "LOR"), "&&": (3, "LAND"), "|": (4, "BOR"), "^": (5, "BXOR"), "&": (6, "BAND"),
    "==": (7, "EQ"), "!=": (7, "NE"), "<": (8, "LT"), "<=": (8, "LE"), ">": (8, "GT"), ">=": (8, "GE"),
    "<<": (9, "SHL"), ">>": (9, "SHR"), "+": (10, "ADD"), "-": (10, "SUB"),
    "*": (11, "MUL"), "/": (11, "DIV"), "%": (11, "MOD"),
}
_ARITH = {"ADD", "SUB", "MUL", "DIV", "MOD", "BAND", "BXOR", "BOR"}
_TOKEN = re.compile(r"\s*(?:(0[xX][0-9a-fA-F]+[uUlL]*|[0-9]+[uUlL]*)|([A-Za-z_][A-Za-z_0-9]*)|"
                    r"(<<|>>|<=|>=|==|!=|&&|\|\||[-+*/%<>!~&|^()?:]))")


class ExprError(ValueError):
    pass


def _tokens(s: str) -> List[Tuple[str, str]]:
    out, pos = [], 0
    s = s.rstrip()
    while pos < len(s):
        m = _TOKEN.match(s, pos)
        if not m or m.end() == pos:
            raise ExprError(f"cannot parse {s[pos:]!r} in {s!r}")
        pos = m.end()
        if m.group(1):
            out.append(("num", m.group(1)))
        elif m.group(2):
            out.append(("id", m.group(2)))
        else:
            out.append(("op", m.group(3)))
    out.append(("end", ""))
    return out


def _literal(text: str) -> Tuple[int, bool]:
    """(value, is_long) of a C integer literal; unsigned ones are refused."""
    body = text.rstrip("uUlL")
    suffix = text[len(body):].lower()
    if "u" in suffix:
        raise ExprError(f"unsigned literal {text} is not supported")
    if body.lower().startswith("0x"):
        v, decimal = int(body, 16), False
    elif len(body) > 1 and body.startswith("0"):
        v, decimal = int(body, 8), False
    else:
        v, decimal = int(body), True
    long_ = "l" in suffix
    if v <= INT_MAX and not long_:
        return v, False
    if not decimal and v <= 0xFFFFFFFF and not long_:
        raise ExprError(f"literal {text} would be unsigned int in C")
    if v <= LONG_MAX:
        return v, True
    raise ExprError(f"literal {text} does not fit a long")


class _Parser:
    """Precedence climbing over C's integer operators; each node is
    (code, is_long) with code a list of (op, arg)."""

    def __init__(self, text: str, variables):
        self.t = _tokens(text)
        self.i = 0
        self.vars = variables
        self.text = text

    def peek(self):
        return self.t[self.i]

    def take(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect(self, op):
        tok = self.take()
        if tok != ("op", op):
            raise ExprError(f"expected {op!r} in {self.text!r}")

    def parse(self):
        code, _ = self.cond()
        if self.peek()[0] != "end":
            raise ExprError(f"trailing {self.peek()[1]!r} in {self.text!r}")
        return code

    def cond(self):
        c, cl = self.binary(1)
        if self.peek() == ("op", "?"):
            self.take()
            a, al = self.cond()
            self.expect(":")
            b, bl = self.cond()
            return c + a + b + [(OP["COND"], 0)], al or bl
        return c, cl

    def binary(self, min_prec):
        lhs, ll = self.unary()
        while True:
            tok = self.peek()
            if tok[0] != "op" or tok[1] not in _BINARY:
                return lhs, ll
            prec, name = _BINARY[tok[1]]
            if prec < min_prec:
                return lhs, ll
            self.take()
            rhs, rl = self.binary(prec + 1)
            if name in ("LAND", "LOR") or name in ("LT", "LE", "GT", "GE", "EQ", "NE"):
                lhs, ll = lhs + rhs + [(OP[name], 0)], False
            elif name in ("SHL", "SHR"):
                lhs = lhs + rhs + [(OP[name] | (0 if ll else WRAP32), 0)]
            else:
                lng = ll or rl
                lhs, ll = lhs + rhs + [(OP[name] | (0 if lng else WRAP32), 0)], lng

    def unary(self):
        tok = self.peek()
        if tok[0] == "op" and tok[1] in ("-", "+", "!", "~"):
            self.take()
            c, lng = self.unary()
            if tok[1] == "+":
                return c, lng
            if tok[1] == "!":
                return c + [(OP["NOT"], 0)], False
            name = "NEG" if tok[1] == "-" else "BNOT"
            return c + [(OP[name] | (0 if lng else WRAP32), 0)], lng
        return self.primary()

    def primary(self):
        kind, text = self.take()
        if kind == "num":
            v, lng = _literal(text)
            return [(OP["CONST"], v)], lng
        if kind == "id":
            idx = self.vars(text)
            if idx is None:
                raise ExprError(f"unknown name {text!r} in {self.text!r}")
            return [(OP["VAR"], idx)], False
        if (kind, text) == ("op", "("):
            c = self.cond()
            self.expect(")")
            return c
        raise ExprError(f"unexpected {text!r} in {self.text!r}")


def _depth(code) -> int:
    d = best = 0
    for op, _ in code:
        o = op & 0x7F
        if o in (OP["CONST"], OP["VAR"]):
            d += 1
        elif o in (OP["NEG"], OP["NOT"], OP["BNOT"]):
            pass
        elif o == OP["COND"]:
            d -= 2
        else:
            d -= 1
        best = max(best, d)
    return best


def compile_expr(text: str, kind: str = "f", num_edges: int = 0,
                 allowed_edges: Optional[Sequence[int]] = None) -> List[Tuple[int, int]]:
    """Program of a node / edge predicate (kind "f": the variable is f) or of
    a filter (kind "e": e0 .. e{num_edges-1}, restricted to allowed_edges)."""
    text = str(text)

    def variables(name):
        if kind == "f":
            return 0 if name == "f" else None
        m = re.fullmatch(r"e(\d+)", name)
        if not m:
            return None
        i = int(m.group(1))
        if i >= num_edges or (allowed_edges is not None and i not in allowed_edges):
            raise ExprError(f"filter names {name}, which is not a matched edge of this motif")
        return i

    code = _Parser(text, variables).parse()
    if len(code) > PROG_MAX:
        raise ExprError(f"expression {text!r} needs {len(code)} instructions (max {PROG_MAX})")
    if _depth(code) > PROG_STACK:
        raise ExprError(f"expression {text!r} is nested too deeply")
    return code


def _wrap32(x: int) -> int:
    return ((x + (1 << 31)) & 0xFFFFFFFF) - (1 << 31)


def _wrap64(x: int) -> int:
    return ((x + (1 << 63)) & 0xFFFFFFFFFFFFFFFF) - (1 << 63)


def evaluate(code, variables: Sequence[int]) -> int:
    """Host interpreter of a program (the device one follows the same rules)."""
    st: List[int] = []
    for op, arg in code:
        o, w = op & 0x7F, bool(op & WRAP32)
        if o == OP["CONST"]:
            st.append(int(arg))
            continue
        if o == OP["VAR"]:
            st.append(int(variables[arg]))
            continue
        if o in (OP["NEG"], OP["NOT"], OP["BNOT"]):
            a = st.pop()
            r = -a if o == OP["NEG"] else (int(a == 0) if o == OP["NOT"] else ~a)
        elif o == OP["COND"]:
            b, a, c = st.pop(), st.pop(), st.pop()
            r = a if c else b
        else:
            b, a = st.pop(), st.pop()
            if o == OP["ADD"]:
                r = a + b
            elif o == OP["SUB"]:
                r = a - b
            elif o == OP["MUL"]:
                r = a * b
            elif o in (OP["DIV"], OP["MOD"]):
                if b == 0:
                    r = 0
                else:
                    q = abs(a) // abs(b)
                    q = q if (a >= 0) == (b >= 0) else -q
                    r = q if o == OP["DIV"] else a - q * b
            elif o == OP["SHL"]:
                r = a << (b & (31 if w else 63))
            elif o == OP["SHR"]:
                r = a >> (b & (31 if w else 63))
            elif o == OP["LT"]:
                r = int(a < b)
            elif o == OP["LE"]:
                r = int(a <= b)
            elif o == OP["GT"]:
                r = int(a > b)
            elif o == OP["GE"]:
                r = int(a >= b)
            elif o == OP["EQ"]:
                r = int(a == b)
            elif o == OP["NE"]:
                r = int(a != b)
            elif o == OP["BAND"]:
                r = a & b
            elif o == OP["BXOR"]:
                r = a ^ b
            elif o == OP["BOR"]:
                r = a | b
            elif o == OP["LAND"]:
                r = int(a != 0 and b != 0)
            elif o == OP["LOR"]:
                r = int(a != 0 or b != 0)
            else:
                raise ExprError(f"bad opcode {op}")
        st.append(_wrap32(r) if w else _wrap64(r))
    return st[-1] if st else 1

"""Run the reference's own multigrid Fortran source on the CPU, to pin the oracle.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (hydro3d_b200) imports this
module.  It exists because the reference (Hydro3D v7.0, fixed-form Fortran
built with `mpiifort -real-size 64`, src_v70/makefile:2-3) cannot be compiled
in this image: there is no Fortran compiler and no MPI.

What it does: a mechanical translator reads the reference's source files as
they lie in the reference tree (they are never copied into this repository),
translates the subset of fixed-form Fortran those files use into Python
functions, and runs them on one emulated MPI rank.  `tests/golden/
make_golden.py` uses it to write golden input/output fixtures that the
oracle and the CUDA path are then checked against bit for bit.

Translated from the reference, statement by statement, with Fortran
semantics:
  * module declarations: module_vars.for (module vars), module_multidata.for
    (type multidom, dom, rdiv, rdv, dom_id, dom_ad, dom_indid), module_mpi.for;
  * set-up: localparameters.for (pl, isp..kep, ttc, rdv, nwork/cof sizing,
    ngg/ngc/nge);
  * the solver: mgsolver.for (coeff, mgkcyc, mgrelax, mgrestr, mgcorr,
    mgbound) and exchangepp.for (exchangepp, exchbc_mgpp);
  * the projection: press.for (calmas, calvel, pbound), exchange.for
    (exchange, exchange_smlvl) and exchange_bc.for (exchange_bc);
  * the SIP solver: sipsol.for (sipsol).
Fortran semantics kept: default REAL and real literals are 8-byte (the
reference's -real-size 64); integer division truncates toward zero; integer
MOD takes the dividend's sign; assignment of a real to an integer truncates;
DO loops evaluate their bounds once and leave the variable at first + trip
count x step; expressions are evaluated left to right as written, every
operation rounded to double (no fused multiply-add); every array access is
bounds checked against the declared or allocated extents.
Array allocations the driver makes itself (the part of initial.for:140-290
that sizes pp, su, sup, dens, dens_mg, faz and the exchange buffers) are
restated in `Reference.__init__` below with their citations.

MPI on one rank: MPI_BARRIER is a no-op and MPI_ALLREDUCE copies its send
buffer into its receive buffer; the point-to-point calls are only reached
when two blocks live on different ranks, which never happens here, so they
raise.
"""
from __future__ import annotations

import math
import os
import re
from typing import Dict, List, Optional, Tuple

import numpy as np

# Directory holding the reference's src_v70 Fortran files.  There is no
# default: the translator runs only where H3D_REFERENCE_SRC names that tree.
REF_SRC = os.environ.get("H3D_REFERENCE_SRC", "")

# ---------------------------------------------------------------------------
# Run-time support used by the generated code
# ---------------------------------------------------------------------------


class FortranError(RuntimeError):
    pass


class FArray:
    """A Fortran array: column-major storage, per-dimension lower bounds,
    bounds-checked element access."""

    __slots__ = ("d", "lo", "ext", "st", "kind")

    def __init__(self, kind: str, bounds):
        self.kind = kind
        self.lo = [int(b[0]) for b in bounds]
        self.ext = [int(b[1]) - int(b[0]) + 1 for b in bounds]
        if any(e < 0 for e in self.ext):
            self.ext = [max(e, 0) for e in self.ext]
        st, n = [], 1
        for e in self.ext:
            st.append(n)
            n *= e
        self.st = st
        fill = {"i": 0, "r": float("nan"), "l": False, "d": None}[kind]
        self.d = [fill] * n

    def _off(self, ix):
        if len(ix) != len(self.lo):
            raise FortranError("rank mismatch")
        off = 0
        for i, lo, e, s in zip(ix, self.lo, self.ext, self.st):
            k = i - lo
            if k < 0 or k >= e:
                raise FortranError("index %r out of bounds lo=%r ext=%r" % (ix, self.lo, self.ext))
            off += k * s
        return off

    def g(self, *ix):
        return self.d[self._off(ix)]

    def s(self, v, *ix):
        self.d[self._off(ix)] = v

    def fill(self, v):
        self.d = [v] * len(self.d)


class Obj:
    """An instance of a derived type (type multidom)."""

    def __init__(self, comps):
        for name, sym in comps.items():
            if sym.rank and not sym.alloc:
                setattr(self, "c_" + name, FArray(sym.kind, [(1, d) for d in sym.dims]))
            elif sym.rank:
                setattr(self, "c_" + name, None)
            else:
                setattr(self, "c_" + name, {"i": 0, "r": 0.0, "l": False, "c": ""}[sym.kind])


class Module:
    pass


def _idiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _imod(a, b):
    return a - b * _idiv(a, b)


def _mod(a, b):
    if isinstance(a, int) and isinstance(b, int):
        return _imod(a, b)
    return math.fmod(a, b)


def _nint(x):
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _sign(a, b):
    return abs(a) if b >= 0 else -abs(a)


def _trip(a, b, s):
    return max(_idiv(b - a + s, s), 0)


def _split_last_paren(ent):
    """'a%b(x,y)' -> ('a%b', ['x', 'y'])."""
    if not ent.endswith(")"):
        raise FortranError("allocate entity %r" % ent)
    depth = 0
    for i in range(len(ent) - 1, -1, -1):
        if ent[i] == ")":
            depth += 1
        elif ent[i] == "(":
            depth -= 1
            if depth == 0:
                return ent[:i], _split_top(ent[i + 1:-1])
    raise FortranError("unbalanced %r" % ent)


def _unreachable(name):
    raise FortranError("%s reached: the single-rank emulation has no peer to talk to" % name)


# ---------------------------------------------------------------------------
# Source reading (fixed form)
# ---------------------------------------------------------------------------


def _strip_comment(t: str) -> str:
    q = None
    for i, c in enumerate(t):
        if q:
            if c == q:
                q = None
        elif c in "'\"":
            q = c
        elif c == "!":
            return t[:i]
    return t


def _split_semicolons(t: str) -> List[str]:
    out, q, cur = [], None, []
    for c in t:
        if q:
            if c == q:
                q = None
            cur.append(c)
        elif c in "'\"":
            q = c
            cur.append(c)
        elif c == ";":
            out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
    out.append("".join(cur))
    return [s for s in out if s.strip()]


def read_statements(path: str) -> List[Tuple[int, str, str]]:
    """Logical statements (line, label, lower-cased text) of a fixed-form file.

    Columns 1-5 label, column 6 continuation, 7-72 statement; a tab in the
    first six columns starts the statement field (a digit after it marks a
    continuation line)."""
    stmts: List[List] = []
    with open(path, encoding="latin-1") as f:
        lines = f.read().split("\n")
    for no, line in enumerate(lines, 1):
        line = line.replace("\r", "")
        if not line.strip() or line[0] in "cC*!" or line.lstrip().startswith("!"):
            continue
        p = 0
        while p < len(line) and p < 6 and line[p] != "\t":
            p += 1
        if p < 6 and p < len(line) and line[p] == "\t":
            head, rest = line[:p], line[p + 1:]
            if not head.strip() and rest[:1] in tuple("123456789"):
                cont, text = True, rest[1:]
            else:
                cont, text = False, rest
        else:
            head, c6, text = line[:5], line[5:6], line[6:]
            cont = c6 not in ("", " ", "0")
        text = _strip_comment(text[:66]).replace("\t", " ")
        label = head.strip()
        if cont:
            if not stmts:
                raise FortranError("%s:%d continuation of nothing" % (path, no))
            stmts[-1][2] += text
            continue
        if not text.strip() and not label:
            continue
        stmts.append([no, label, text])
    out = []
    for no, label, text in stmts:
        parts = _split_semicolons(text)
        for k, p in enumerate(parts):
            out.append((no, label if k == 0 else "", p.strip().lower()))
        if not parts and label:
            out.append((no, label, "continue"))
    return out


# ---------------------------------------------------------------------------
# Expressions
# ---------------------------------------------------------------------------

_TOK = re.compile(r"""
   (?P<num>(\d+\.(?![a-z]+\.)\d*|\.\d+|\d+)([ed][+-]?\d+)?)
 | (?P<dot>\.(eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv|true|false)\.)
 | (?P<name>[a-z_][a-z0-9_]*)
 | (?P<str>'[^']*'|"[^"]*")
 | (?P<op>\*\*|//|==|/=|<=|>=|=>|[-+*/(),%<>=:])
""", re.X)


def tokenize(s: str):
    s = s.replace(" ", "").replace("\t", "")
    pos, out = 0, []
    while pos < len(s):
        m = _TOK.match(s, pos)
        if not m:
            raise FortranError("cannot tokenize %r at %r" % (s, s[pos:]))
        kind = m.lastgroup
        out.append((kind, m.group(0)))
        pos = m.end()
    return out


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.p = 0

    def peek(self, k=0):
        return self.t[self.p + k] if self.p + k < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise FortranError("expected %r got %r in %r" % (val, tok, self.t))
        self.p += 1
        return tok

    def done(self):
        return self.p >= len(self.t)

    def expr(self):
        return self.or_()

    def or_(self):
        a = self.and_()
        while self.peek()[1] in (".or.",):
            self.take()
            a = ("or", a, self.and_())
        return a

    def and_(self):
        a = self.not_()
        while self.peek()[1] == ".and.":
            self.take()
            a = ("and", a, self.not_())
        return a

    def not_(self):
        if self.peek()[1] == ".not.":
            self.take()
            return ("not", self.not_())
        return self.rel()

    _REL = {".eq.": "==", "==": "==", ".ne.": "!=", "/=": "!=", ".lt.": "<", "<": "<",
            ".le.": "<=", "<=": "<=", ".gt.": ">", ">": ">", ".ge.": ">=", ">=": ">="}

    def rel(self):
        a = self.add()
        op = self.peek()[1]
        if op in self._REL:
            self.take()
            return ("rel", self._REL[op], a, self.add())
        return a

    def add(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = self.mul()
            a = ("neg", a) if op == "-" else a
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.pow_()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = ("bin", op, a, self.pow_())
        return a

    def pow_(self):
        a = self.primary()
        if self.peek()[1] == "**":
            self.take()
            if self.peek()[1] == "-":
                self.take()
                b = ("neg", self.pow_())
            else:
                b = self.pow_()
            return ("bin", "**", a, b)
        return a

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            if re.fullmatch(r"\d+", val):
                return ("int", int(val))
            return ("real", float(val.replace("d", "e")))
        if kind == "dot" and val in (".true.", ".false."):
            self.take()
            return ("bool", val == ".true.")
        if kind == "str":
            self.take()
            return ("str", val[1:-1])
        if val == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return e
        if kind == "name":
            return self.designator()
        if val in ("+", "-"):
            self.take()
            e = self.pow_()
            return ("neg", e) if val == "-" else e
        raise FortranError("unexpected %r in %r" % (val, self.t))

    def args(self):
        self.take("(")
        out = []
        if self.peek()[1] == ")":
            self.take()
            return out
        while True:
            if self.peek()[1] == ":" or (self.peek()[1] != ")" and self.peek(1)[1] == ":"):
                lo = None if self.peek()[1] == ":" else self.expr()
                self.take(":")
                hi = None if self.peek()[1] in (",", ")") else self.expr()
                out.append(("range", lo, hi))
            else:
                out.append(self.expr())
            if self.peek()[1] == ",":
                self.take()
                continue
            self.take(")")
            return out

    def designator(self):
        name = self.take()[1]
        node = ("name", name, self.args() if self.peek()[1] == "(" else None)
        while self.peek()[1] == "%":
            self.take()
            comp = self.take()[1]
            node = ("comp", node, comp, self.args() if self.peek()[1] == "(" else None)
        return node


def parse_expr(s: str):
    p = Parser(tokenize(s))
    e = p.expr()
    if not p.done():
        raise FortranError("trailing tokens in %r" % s)
    return e


# ---------------------------------------------------------------------------
# Declarations
# ---------------------------------------------------------------------------


class Sym:
    def __init__(self, kind, dims=(), alloc=False, const=None, dtype=None):
        self.kind = kind          # i r l c d
        self.dims = list(dims)    # declared extents (expressions as text) or [] for deferred
        self.rank = len(dims)
        self.alloc = alloc        # allocatable / pointer (deferred shape)
        self.const = const
        self.dtype = dtype


def _split_top(s: str, sep=","):
    out, depth, cur, q = [], 0, [], None
    for c in s:
        if q:
            cur.append(c)
            if c == q:
                q = None
            continue
        if c in "'\"":
            q = c
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        if c == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
    out.append("".join(cur))
    return [x.strip() for x in out if x.strip()]


_DECL = re.compile(r"^(integer|double\s*precision|real(\s*\(\s*kind\s*=\s*\d+\s*\)|\s*\*\s*\d+)?|logical|"
                   r"character(\s*\(\s*\d+\s*\)|\*\d+)?|type\s*\(\s*\w+\s*\))(?=\s|,|::)\s*(.*)$")


def parse_decl(text: str):
    """-> list of (name, Sym) or None if the statement is not a declaration."""
    m = _DECL.match(text)
    if not m:
        return None
    base = m.group(1).replace(" ", "")
    rest = m.group(len(m.groups()))
    if base.startswith("integer"):
        kind = "i"
    elif base.startswith("double") or base.startswith("real"):
        kind = "r"                       # -real-size 64: default REAL is 8 bytes
    elif base.startswith("logical"):
        kind = "l"
    elif base.startswith("character"):
        kind = "c"
    else:
        kind = "d"
    dtype = re.match(r"type\((\w+)\)", base).group(1) if kind == "d" else None
    attrs, ents = "", rest
    if "::" in rest:
        attrs, ents = rest.split("::", 1)
    elif rest.startswith(","):
        raise FortranError("declaration without :: %r" % text)
    alloc, dims, param = False, None, False
    for a in _split_top(attrs.lstrip(",")):
        a = a.replace(" ", "")
        if a in ("allocatable", "pointer", "target", "save"):
            alloc = alloc or a in ("allocatable", "pointer")
        elif a.startswith("dimension("):
            dims = _split_top(a[len("dimension("):-1])
        elif a == "parameter":
            param = True
        elif a.startswith("intent"):
            pass
        else:
            raise FortranError("attribute %r" % a)
    out = []
    for e in _split_top(ents):
        e = e.replace(" ", "")
        const = None
        if "=" in e and not e.startswith("=>"):
            e, init = e.split("=", 1)
            if param:
                const = init
        m2 = re.match(r"^(\w+)(\((.*)\))?$", e)
        if not m2:
            raise FortranError("entity %r" % e)
        name = m2.group(1)
        d = _split_top(m2.group(3)) if m2.group(3) else dims
        d = d or []
        deferred = all(x == ":" for x in d) and bool(d)
        out.append((name, Sym(kind, d, alloc or deferred, const, dtype)))
    return out


# ---------------------------------------------------------------------------
# Translation of subroutines
# ---------------------------------------------------------------------------

_INTRINSIC = {"mod", "max", "min", "abs", "sqrt", "real", "dble", "int", "nint", "float", "sign", "log", "exp"}


class Unit:
    def __init__(self, name, args, body, path):
        self.name, self.args, self.body, self.path = name, args, body, path


class Translator:
    """Holds module symbols and translates subroutines into Python source."""

    def __init__(self):
        self.mod: Dict[str, Sym] = {}
        self.types: Dict[str, Dict[str, Sym]] = {}
        self.units: Dict[str, Unit] = {}
        self.params: Dict[str, str] = {}

    # -- modules ------------------------------------------------------------
    def load_module_file(self, path):
        stmts = read_statements(path)
        in_type, in_contains = None, False
        for no, label, t in stmts:
            if in_contains:
                if re.match(r"^end\s*module", t):
                    in_contains = False
                continue
            if re.match(r"^module\s+\w+$", t):
                continue
            if re.match(r"^end\s*module", t) or t in ("save", "implicit none") or t.startswith("include"):
                continue
            if t == "contains":
                in_contains = True
                continue
            m = re.match(r"^type\s+(\w+)$", t)
            if m:
                in_type = m.group(1)
                self.types[in_type] = {}
                continue
            if re.match(r"^end\s*type", t):
                in_type = None
                continue
            d = parse_decl(t)
            if d is None:
                raise FortranError("%s:%d unexpected in module: %r" % (path, no, t))
            for name, sym in d:
                if in_type:
                    self.types[in_type][name] = sym
                else:
                    self.mod[name] = sym
                    if sym.const is not None:
                        self.params[name] = sym.const

    # -- subroutines --------------------------------------------------------
    def load_units(self, path, names):
        stmts = read_statements(path)
        i = 0
        while i < len(stmts):
            no, label, t = stmts[i]
            m = re.match(r"^subroutine\s+(\w+)\s*(\((.*)\))?$", t)
            if m:
                name = m.group(1)
                args = [a.strip() for a in (m.group(3) or "").split(",") if a.strip()]
                j = i + 1
                while not re.match(r"^end(\s*subroutine.*)?$", stmts[j][2]):
                    j += 1
                if name in names:
                    self.units[name] = Unit(name, args, stmts[i + 1:j], path)
                i = j + 1
                continue
            i += 1
        missing = set(names) - set(self.units)
        if missing:
            raise FortranError("subroutines not found in %s: %s" % (path, sorted(missing)))

    def translate_all(self):
        src = ["# generated from the reference's Fortran by oracle/fortran_ref.py", ""]
        for u in self.units.values():
            src += UnitTranslator(self, u).translate()
            src.append("")
        return "\n".join(src)


class UnitTranslator:
    def __init__(self, tr: Translator, unit: Unit):
        self.tr, self.u = tr, unit
        self.loc: Dict[str, Sym] = {}
        self.out: List[str] = []
        self.ind = 1
        self.labels: List[str] = []

    # -- symbols -----------------------------------------------------------
    def sym(self, name) -> Tuple[str, Sym]:
        if name in self.loc:
            return "v_" + name, self.loc[name]
        if name in self.tr.mod:
            return "M.v_" + name, self.tr.mod[name]
        raise FortranError("%s: undeclared %r" % (self.u.name, name))

    # -- expressions -> (code, kind) ---------------------------------------
    def ex(self, e) -> Tuple[str, str]:
        k = e[0]
        if k == "int":
            return str(e[1]), "i"
        if k == "real":
            return repr(e[1]), "r"
        if k == "bool":
            return repr(e[1]), "l"
        if k == "str":
            return repr(e[1]), "c"
        if k == "neg":
            c, t = self.ex(e[1])
            return "(-%s)" % c, t
        if k == "bin":
            op = e[1]
            a, ta = self.ex(e[2])
            b, tb = self.ex(e[3])
            if ta in "lc" or tb in "lc":
                raise FortranError("arithmetic on %s/%s" % (ta, tb))
            if ta == "i" and tb == "i":
                if op == "/":
                    return "_idiv(%s, %s)" % (a, b), "i"
                return "(%s %s %s)" % (a, op, b), "i"
            if op == "**":
                if tb != "i":
                    raise FortranError("real exponent")
                # x**n with an integer n: repeated multiplication
                return "_rpow(%s, %s)" % (a, b), "r"
            return "(%s %s %s)" % (a, op, b), "r"
        if k == "rel":
            a, _ = self.ex(e[2])
            b, _ = self.ex(e[3])
            return "(%s %s %s)" % (a, e[1], b), "l"
        if k in ("and", "or"):
            a, _ = self.ex(e[1])
            b, _ = self.ex(e[2])
            return "(%s %s %s)" % (a, k, b), "l"
        if k == "not":
            a, _ = self.ex(e[1])
            return "(not %s)" % a, "l"
        if k == "name":
            return self.name_ref(e)
        if k == "comp":
            return self.comp_ref(e)
        raise FortranError("expr %r" % (e,))

    def intrinsic(self, name, args):
        cs = [self.ex(a) for a in args]
        codes = [c for c, _ in cs]
        kinds = [t for _, t in cs]
        if name == "mod":
            return ("_imod(%s, %s)" % tuple(codes), "i") if kinds == ["i", "i"] else \
                ("math.fmod(%s, %s)" % tuple(codes), "r")
        if name in ("max", "min"):
            t = "i" if all(x == "i" for x in kinds) else "r"
            inner = ", ".join(codes if t == "i" else ["float(%s)" % c for c in codes])
            return "%s(%s)" % (name, inner), t
        if name == "abs":
            return "abs(%s)" % codes[0], kinds[0]
        if name == "sqrt":
            return "math.sqrt(%s)" % codes[0], "r"
        if name in ("log", "exp"):
            return "math.%s(%s)" % (name, codes[0]), "r"
        if name in ("real", "dble", "float"):
            return "float(%s)" % codes[0], "r"
        if name == "int":
            return "int(%s)" % codes[0], "i"
        if name == "nint":
            return "_nint(%s)" % codes[0], "i"
        if name == "sign":
            return "_sign(%s, %s)" % tuple(codes), kinds[0]
        raise FortranError(name)

    def name_ref(self, e):
        _, name, args = e
        if name in self.tr.params and name not in self.loc:
            return self.ex(parse_expr(self.tr.params[name]))
        if args is not None and name not in self.loc and name not in self.tr.mod:
            if name in _INTRINSIC:
                return self.intrinsic(name, args)
            raise FortranError("%s: unknown function %r" % (self.u.name, name))
        code, sym = self.sym(name)
        if args is None:
            return code, sym.kind if not sym.rank else "A"
        return "%s.g(%s)" % (code, ", ".join(self.ex(a)[0] for a in args)), sym.kind

    def comp_sym(self, e) -> Sym:
        """Symbol of the object a comp node's base refers to."""
        base = e[1]
        if base[0] == "name":
            _, s = self.sym(base[1])
        else:
            s = self.comp_sym(base)
        if s.kind != "d":
            raise FortranError("component of non-derived %r" % (base,))
        return self.tr.types[s.dtype][e[2]]

    def comp_ref(self, e):
        _, base, comp, args = e
        bcode, bkind = self.ex(base)
        s = self.comp_sym(e)
        code = "%s.c_%s" % (bcode, comp)
        if args is None:
            return code, s.kind if not s.rank else "A"
        return "%s.g(%s)" % (code, ", ".join(self.ex(a)[0] for a in args)), s.kind

    # -- statements ---------------------------------------------------------
    def emit(self, line):
        self.out.append("    " * self.ind + line)

    def lhs(self, e):
        """-> (kind, setter template with {v}, is_whole_array)."""
        if e[0] == "name":
            _, name, args = e
            code, sym = self.sym(name)
            if args is None:
                if sym.rank:
                    return sym.kind, "%s.fill({v})" % code, True
                return sym.kind, "%s = {v}" % code, False
            idx = ", ".join(self.ex(a)[0] for a in args)
            return sym.kind, "%s.s({v}, %s)" % (code, idx), False
        if e[0] == "comp":
            _, base, comp, args = e
            bcode, _ = self.ex(base)
            s = self.comp_sym(e)
            code = "%s.c_%s" % (bcode, comp)
            if args is None:
                if s.rank:
                    return s.kind, "%s.fill({v})" % code, True
                return s.kind, "%s = {v}" % code, False
            idx = ", ".join(self.ex(a)[0] for a in args)
            return s.kind, "%s.s({v}, %s)" % (code, idx), False
        raise FortranError("lhs %r" % (e,))

    @staticmethod
    def convert(code, src, dst):
        if dst == "i" and src == "r":
            return "int(%s)" % code
        if dst == "r" and src == "i":
            return "float(%s)" % code
        return code

    def assign(self, t):
        lhs_s, rhs_s = self.split_assign(t)
        if rhs_s is None:
            raise FortranError("not an assignment: %r" % t)
        lhs = Parser(tokenize(lhs_s)).designator()
        kind, tmpl, whole = self.lhs(lhs)
        code, k = self.ex(parse_expr(rhs_s))
        self.emit(tmpl.format(v=self.convert(code, k, kind)))

    @staticmethod
    def split_assign(t):
        depth = 0
        for i, c in enumerate(t):
            if c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
            elif c == "=" and depth == 0:
                prev = t[i - 1] if i else ""
                nxt = t[i + 1] if i + 1 < len(t) else ""
                if prev in "<>=/" or nxt in "=>":
                    continue
                return t[:i], t[i + 1:]
        return t, None

    @staticmethod
    def paren_split(t):
        """'(cond) rest' -> (cond, rest)."""
        t = t.strip()
        if not t.startswith("("):
            raise FortranError("expected ( in %r" % t)
        depth = 0
        for i, c in enumerate(t):
            if c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
                if depth == 0:
                    return t[1:i], t[i + 1:].strip()
        raise FortranError("unbalanced %r" % t)

    def call(self, t):
        m = re.match(r"^call\s*(\w+)\s*(\((.*)\))?$", t)
        name = m.group(1)
        args = _split_top(m.group(3)) if m.group(3) else []
        if name == "mpi_barrier":
            self.emit("pass")
            return
        if name == "mpi_allreduce":
            src, dst, cnt = args[0], args[1], args[2]
            sk, stmpl, sw = self.lhs(Parser(tokenize(dst)).designator())
            scode, skind = self.ex(parse_expr(src))
            if sw:
                self.emit("%s.d = list(%s.d)" % (stmpl.split(".fill")[0], scode))
            else:
                self.emit(stmpl.format(v=self.convert(scode, skind, sk)))
            return
        if name.startswith("mpi_"):
            self.emit("_unreachable(%r)" % name)
            return
        if name not in self.tr.units:
            self.emit("_unreachable(%r)" % ("call " + name))
            return
        callee = self.tr.units[name]
        vals = [self.ex(parse_expr(a))[0] for a in args]
        self.emit("%s(%s)" % (name, ", ".join(vals)))
        # Fortran passes by reference: refuse callees that assign a dummy argument
        for a in callee.args:
            for _, _, s in callee.body:
                l, r = self.split_assign(s)
                if r is not None and re.fullmatch(r"%s(\(.*\))?" % a, l.replace(" ", "")):
                    raise FortranError("%s assigns its argument %s" % (name, a))

    def allocate(self, t, dealloc=False):
        inner, rest = self.paren_split(t[len("deallocate" if dealloc else "allocate"):].strip())
        for ent in _split_top(inner):
            if dealloc:
                d = Parser(tokenize(ent)).designator()
                kind, tmpl, whole = self.lhs(d)
                self.emit(tmpl.replace(".fill({v})", " = None") if whole else "pass")
                continue
            target, dims = _split_last_paren(ent.replace(" ", ""))
            bounds = []
            for dd in dims:
                parts = _split_top(dd, ":")
                lo, hi = (parts[0], parts[1]) if len(parts) == 2 else ("1", parts[0])
                bounds.append("(%s, %s)" % (self.ex(parse_expr(lo))[0], self.ex(parse_expr(hi))[0]))
            d = Parser(tokenize(target)).designator()
            if d[0] == "name":
                code, sym = self.sym(d[1])
            else:
                code = self.ex(d[1])[0] + ".c_" + d[2]
                sym = self.comp_sym(d)
            self.emit("%s = FArray(%r, [%s])" % (code, sym.kind, ", ".join(bounds)))

    def block(self, stmts, i, stop_words):
        """Translate statements from i until one whose text matches stop_words;
        returns the index of that statement."""
        start_len = len(self.out)
        while i < len(stmts):
            no, label, t = stmts[i]
            if any(re.match(w, t) for w in stop_words):
                break
            if label and self.in_dispatch and self.ind == self.top_ind and label in self.labels:
                self.emit("_lab = %s" % label)
                self.ind -= 1
                self.emit("if _lab == %s:" % label)
                self.ind += 1
            i = self.statement(stmts, i)
        if len(self.out) == start_len:
            self.emit("pass")
        return i

    def statement(self, stmts, i):
        no, label, t = stmts[i]
        try:
            return self._statement(stmts, i)
        except FortranError as e:
            raise FortranError("%s:%d (%s): %s" % (os.path.basename(self.u.path), no, t, e)) from None

    def _statement(self, stmts, i):
        no, label, t = stmts[i]
        if t in ("continue", "return") or t.startswith(("print", "write", "format", "use ", "implicit")):
            if t == "return":
                self.emit("return")
            return i + 1
        if t == "stop" or t.startswith("stop"):
            self.emit("raise FortranError('stop at line %d')" % no)
            return i + 1
        d = parse_decl(t)
        if d is not None:
            return i + 1
        m = re.match(r"^do\s+(\w+)\s*=(.*)$", t)
        if m:
            var = m.group(1)
            parts = _split_top(m.group(2))
            a, b = self.ex(parse_expr(parts[0]))[0], self.ex(parse_expr(parts[1]))[0]
            s = self.ex(parse_expr(parts[2]))[0] if len(parts) > 2 else "1"
            vcode, _ = self.sym(var)
            self.tmp += 1
            n = "_n%d" % self.tmp
            a0 = "_a%d" % self.tmp
            self.emit("%s = %s; %s = _trip(%s, %s, %s)" % (a0, a, n, a0, b, s))
            self.emit("for %s in range(%s, %s + %s * (%s), %s):" % (vcode, a0, a0, n, s, s))
            self.ind += 1
            self.depth += 1
            j = self.block(stmts, i + 1, [r"^end\s*do$"])
            self.depth -= 1
            self.ind -= 1
            post = "%s = %s + %s * (%s)" % (vcode, a0, n, s)
            if self.in_dispatch:
                # a GOTO out of the loop leaves the DO variable as it is (no
                # final increment) and continues at the label
                self.emit("else:")
                self.ind += 1
                self.emit(post)
                self.ind -= 1
                if self.depth:
                    self.emit("if _brk:")
                    self.ind += 1
                    self.emit("break")
                    self.ind -= 1
                else:
                    self.emit("if _brk:")
                    self.ind += 1
                    self.emit("_brk = False")
                    self.emit("continue")
                    self.ind -= 1
            else:
                self.emit(post)
            return j + 1
        if re.match(r"^do\s+\d", t):
            raise FortranError("unsupported do form")
        if re.match(r"^if\s*\(", t):
            cond, rest = self.paren_split(t[2:])
            c = self.ex(parse_expr(cond))[0]
            if rest == "then":
                self.emit("if %s:" % c)
                self.ind += 1
                j = self.block(stmts, i + 1, [r"^else", r"^end\s*if$"])
                self.ind -= 1
                while True:
                    tj = stmts[j][2]
                    if re.match(r"^end\s*if$", tj):
                        return j + 1
                    m2 = re.match(r"^else\s*if\s*(\(.*)$", tj)
                    if m2:
                        cond2, rest2 = self.paren_split(m2.group(1))
                        if rest2 != "then":
                            raise FortranError("else if without then")
                        self.emit("elif %s:" % self.ex(parse_expr(cond2))[0])
                    else:
                        self.emit("else:")
                    self.ind += 1
                    j = self.block(stmts, j + 1, [r"^else", r"^end\s*if$"])
                    self.ind -= 1
            self.emit("if %s:" % c)
            self.ind += 1
            n0 = len(self.out)
            self.statement([(no, "", rest)], 0)
            if len(self.out) == n0:
                self.emit("pass")
            self.ind -= 1
            return i + 1
        m = re.match(r"^select\s*case\s*\((.*)\)$", t)
        if m:  # SELECT CASE with scalar case values (no ranges)
            self.tmp += 1
            sv = "_sel%d" % self.tmp
            self.emit("%s = %s" % (sv, self.ex(parse_expr(m.group(1)))[0]))
            j, first = i + 1, True
            while True:
                tj = stmts[j][2]
                if re.match(r"^end\s*select$", tj):
                    if first:
                        self.emit("pass")
                    return j + 1
                mc = re.match(r"^case\s*\((.*)\)$", tj)
                if mc:
                    vals = _split_top(mc.group(1))
                    if any(":" in v for v in vals):
                        raise FortranError("case ranges are not supported")
                    cond = " or ".join("%s == %s" % (sv, self.ex(parse_expr(v))[0]) for v in vals)
                    self.emit(("if %s:" if first else "elif %s:") % cond)
                elif re.match(r"^case\s+default$", tj):
                    self.emit("else:" if not first else "if True:")
                else:
                    raise FortranError("statement before the first case")
                first = False
                self.ind += 1
                j = self.block(stmts, j + 1, [r"^case\b", r"^end\s*select$"])
                self.ind -= 1
        m = re.match(r"^go\s*to\s*(\d+)$", t)
        if m:
            self.emit("_lab = %s" % m.group(1))
            if self.depth:  # out of the enclosing DO loops, then to the label
                self.emit("_brk = True")
                self.emit("break")
            else:
                self.emit("continue")
            return i + 1
        if re.match(r"^call\s", t):
            self.call(t)
            return i + 1
        if t.startswith("deallocate"):
            self.allocate(t, dealloc=True)
            return i + 1
        if t.startswith("allocate"):
            self.allocate(t)
            return i + 1
        if "=>" in t:
            l, r = t.split("=>", 1)
            lcode, _, _ = self.lhs(Parser(tokenize(l)).designator())[1], None, None
            rcode, _ = self.ex(parse_expr(r))
            self.emit(lcode.replace(".fill({v})", " = " + rcode).replace(" = {v}", " = " + rcode))
            return i + 1
        self.assign(t)
        return i + 1

    def translate(self):
        u = self.u
        body = u.body
        for no, label, t in body:
            d = parse_decl(t)
            if d:
                for name, sym in d:
                    self.loc[name] = sym
        for a in u.args:
            if a not in self.loc:
                raise FortranError("%s: undeclared dummy %s" % (u.name, a))
        self.tmp = 0
        self.depth = 0
        self.top_ind = -1
        self.labels = [lb for _, lb, _ in body if lb]
        gotos = any(re.match(r"^go\s*to", t) or re.search(r"\)\s*go\s*to", t) for _, _, t in body)
        self.in_dispatch = gotos
        head = ["def %s(%s):" % (u.name, ", ".join("v_" + a for a in u.args))]
        self.out = []
        # automatic arrays (explicit extents in a declaration)
        for name, sym in self.loc.items():
            if sym.rank and not sym.alloc and name not in u.args:
                bounds = []
                for dd in sym.dims:
                    parts = _split_top(dd, ":")
                    lo, hi = (parts[0], parts[1]) if len(parts) == 2 else ("1", parts[0])
                    bounds.append("(%s, %s)" % (self.ex(parse_expr(lo))[0], self.ex(parse_expr(hi))[0]))
                self.emit("v_%s = FArray(%r, [%s])" % (name, sym.kind, ", ".join(bounds)))
        if gotos:
            self.emit("_lab = 0")
            self.emit("_brk = False")
            self.emit("while True:")
            self.ind += 1
            self.emit("if _lab == 0:")
            self.ind += 1
            self.top_ind = self.ind
            self.block(body, 0, [r"^\b\B"])
            self.emit("return")
            self.ind -= 2
        else:
            self.block(body, 0, [r"^\b\B"])
        return head + self.out


def _rpow(x, n):
    if n < 0:
        return 1.0 / _rpow(x, -n)
    r = 1.0
    for _ in range(n):
        r = r * x
    return r


# ---------------------------------------------------------------------------
# The reference, set up for a block layout
# ---------------------------------------------------------------------------

SOLVER_UNITS = {
    "mgsolver.for": ["coeff", "mgkcyc", "mgrelax", "mgrestr", "mgcorr", "mgbound"],
    "exchangepp.for": ["exchangepp", "exchbc_mgpp"],
    "localparameters.for": ["localparameters"],
    "press.for": ["calmas", "calvel", "pbound"],
    "exchange.for": ["exchange", "exchange_smlvl"],
    "exchange_bc.for": ["exchange_bc"],
    "sipsol.for": ["sipsol"],
}
MODULE_FILES = ["module_vars.for", "module_multidata.for", "module_mpi.for"]
MPI_CONSTANTS = {"mpi_comm_world": 0, "mpi_double_precision": 1, "mpi_integer": 2, "mpi_max": 3,
                 "mpi_sum": 4, "mpi_min": 5, "mpi_status_size": 6, "mpi_status_ignore": 0,
                 "mpi_real": 7}


def build_namespace(src_dir: str = REF_SRC):
    tr = Translator()
    for name, val in MPI_CONSTANTS.items():
        tr.mod[name] = Sym("i")
    for f in MODULE_FILES:
        tr.load_module_file(os.path.join(src_dir, f))
    for f, names in SOLVER_UNITS.items():
        tr.load_units(os.path.join(src_dir, f), names)
    code = tr.translate_all()
    M = Module()
    for name, sym in tr.mod.items():
        setattr(M, "v_" + name, None if sym.rank else {"i": 0, "r": 0.0, "l": False, "c": "", "d": None}[sym.kind])
    for name, val in MPI_CONSTANTS.items():
        setattr(M, "v_" + name, val)
    ns = {"M": M, "FArray": FArray, "FortranError": FortranError, "math": math, "_idiv": _idiv,
          "_imod": _imod, "_nint": _nint, "_sign": _sign, "_trip": _trip, "_rpow": _rpow,
          "_unreachable": _unreachable}
    exec(compile(code, "<reference-fortran>", "exec"), ns)
    return tr, M, ns, code


class Reference:
    """The reference's multigrid state for one rank holding all blocks.

    blocks: descriptors with the fields of h3d_block_desc (n, ngrid, h,
    nb_face, nb_corner, nb_edge, nb_periodic, bc, origin).  Domain ids are
    the block indices 0..nblocks-1, all on rank 0."""

    def __init__(self, blocks, ngrd_gl, mg_itrsch=3, irestr=2, iproln=1, pl_ex=0, lsm=False,
                 src_dir: str = REF_SRC):
        self.tr, M, self.ns, self.code = build_namespace(src_dir)
        self.M = M
        nb = len(blocks)
        self.blocks = blocks
        T = self.tr.types["multidom"]
        # module_multidata / alloc_dom.for:319-320,440: domain maps
        M.v_nbp = nb
        M.v_num_domains = nb
        M.v_dom = FArray("d", [(1, nb)])
        M.v_dom_id = FArray("i", [(1, nb)])
        M.v_dom_ad = FArray("i", [(0, nb - 1)])
        M.v_dom_indid = FArray("i", [(0, nb - 1)])
        M.v_rdiv = FArray("i", [(0, nb - 1)])
        M.v_myrank = 0
        M.v_nprocs = 1
        rdivs = [int(getattr(d, "rdiv", 1) or 1) for d in blocks]
        lmr = any(r > 1 for r in rdivs)
        ngrid_input = ngrd_gl - (max(rdivs).bit_length() - 1)
        # control.cin settings the path reads (LMR = 2: local mesh refinement)
        M.v_lmr = 2 if lmr else 1
        M.v_pl_ex = pl_ex
        M.v_ngrid_input = ngrid_input
        M.v_solver = 2
        M.v_mg_itrsch = mg_itrsch
        M.v_irestr = irestr
        M.v_iproln = iproln
        M.v_l_lsm = bool(lsm)
        M.v_l_lsmbase = False
        M.v_periodic = any(int(c) == 5 for d in blocks for c in d.bc)
        # g_dx: the unrefined spacing; a block of ratio rdiv has g_dx / rdiv
        # (localparameters.for:247-249) and its origin in its own cells
        M.v_g_dx, M.v_g_dy, M.v_g_dz = (float(x) * rdivs[0] for x in blocks[0].h)
        for ib, d in enumerate(blocks, 1):
            o = Obj(T)
            M.v_dom.s(o, ib)
            M.v_dom_id.s(ib - 1, ib)
            M.v_dom_ad.s(0, ib - 1)
            M.v_dom_indid.s(ib, ib - 1)
            r = rdivs[ib - 1]
            M.v_rdiv.s(r, ib - 1)
            if tuple(float(x) * r for x in d.h) != (M.v_g_dx, M.v_g_dy, M.v_g_dz):
                raise FortranError("block spacings are not g_dx / rdiv")
            o.c_ngrid = ngrid_input  # localparameters.for:44-47 adds log2(rdiv)
            # alloc_dom.for:read_infodom extents (xsl..zel) and neighbours
            if any(d.origin[a] % r or d.n[a] % r for a in range(3)):
                raise FortranError("refined block not aligned with the unrefined grid")
            o.c_xsl = (d.origin[0] // r) * M.v_g_dx
            o.c_xel = ((d.origin[0] + d.n[0]) // r) * M.v_g_dx
            o.c_ysl = (d.origin[1] // r) * M.v_g_dy
            o.c_yel = ((d.origin[1] + d.n[1]) // r) * M.v_g_dy
            o.c_zsl = (d.origin[2] // r) * M.v_g_dz
            o.c_zel = ((d.origin[2] + d.n[2]) // r) * M.v_g_dz
            for name, v in zip(("iprev", "inext", "jprev", "jnext", "kprev", "knext"), d.nb_face):
                setattr(o, "c_" + name, int(v))
            for name, v in zip(("corprev1", "corprev2", "corprev3", "corprev4",
                                "cornext1", "cornext2", "cornext3", "cornext4"), d.nb_corner):
                setattr(o, "c_" + name, int(v))
            for name, v in zip(["edgprev%d" % k for k in range(1, 7)] + ["edgnext%d" % k for k in range(1, 7)],
                               d.nb_edge):
                setattr(o, "c_" + name, int(v))
            for name, v in zip(("per_ip", "per_in", "per_jp", "per_jn", "per_kp", "per_kn"), d.nb_periodic):
                setattr(o, "c_" + name, int(v))
            for name, v in zip(("bc_west", "bc_east", "bc_south", "bc_north", "bc_bottom", "bc_top"), d.bc):
                setattr(o, "c_" + name, int(v))
        M.v_ngrd_gl = ngrd_gl
        self.ns["localparameters"]()
        if M.v_ngrd_gl != ngrd_gl:
            raise FortranError("ngrd_gl changed by localparameters")
        for ib, d in enumerate(blocks, 1):
            if M.v_dom.g(ib).c_ngrid != int(d.ngrid):
                raise FortranError("block %d: localparameters gives ngrid %d, the descriptor %d"
                                   % (ib - 1, M.v_dom.g(ib).c_ngrid, int(d.ngrid)))
        # initial.for:140-290 allocations of the arrays the solver touches
        for ib in range(1, nb + 1):
            o = M.v_dom.g(ib)
            tti, ttj, ttk = o.c_ttc_i, o.c_ttc_j, o.c_ttc_k
            for f in ("pp", "su", "sup", "dens", "p", "u", "v", "w", "ustar", "vstar", "wstar",
                      "ap", "ae", "aw", "an", "as", "at", "ab"):
                setattr(o, "c_" + f, FArray("r", [(1, tti), (1, ttj), (1, ttk)]))  # initial.for:146-163
            o.c_faz = FArray("i", [(1, ngrd_gl)])                       # initial.for:250
            o.c_stfcinf = FArray("r", [(1, 6), (1, M.v_pl), (1, M.v_ngg)])  # initial.for:183
            for f in ("sendb_m1", "sendb_p1", "recvb_m1", "recvb_p1", "sendb_m2", "sendb_p2",
                      "recvb_m2", "recvb_p2", "sendb_m3", "sendb_p3", "recvb_m3", "recvb_p3"):
                setattr(o, "c_" + f, FArray("r", [(1, M.v_ngg)]))          # initial.for:252-257
            for c in range(1, 5):
                for f in ("sc%dm", "sc%dp", "rc%dm", "rc%dp"):
                    setattr(o, "c_" + f % c, FArray("r", [(1, M.v_ngc)]))  # initial.for:259-266
            for e in range(1, 7):
                for f in ("se%dm", "se%dp", "re%dm", "re%dp"):
                    setattr(o, "c_" + f % e, FArray("r", [(1, M.v_nge)]))  # initial.for:268-279
            if lsm:
                # initial.for:200-215: ijkp_lsm offsets of the per-level densities
                pl = M.v_pl
                o.c_ijkp_lsm = FArray("i", [(0, o.c_ngrid)])
                o.c_ijkp_lsm.fill(0)
                o.c_ijkp_lsm.s((tti - 2 * pl) * (ttj - 2 * pl) * (ttk - 2 * pl), 1)
                for g in range(2, o.c_ngrid + 1):
                    mi = _idiv(o.c_iep - o.c_isp + 1, 2 ** (g - 1)) + 2
                    mj = _idiv(o.c_jep - o.c_jsp + 1, 2 ** (g - 1)) + 2
                    mk = _idiv(o.c_kep - o.c_ksp + 1, 2 ** (g - 1)) + 2
                    o.c_ijkp_lsm.s(o.c_ijkp_lsm.g(g - 1) + (mi - 2) * (mj - 2) * (mk - 2), g)
                o.c_tot = o.c_ijkp_lsm.g(o.c_ngrid)
                o.c_dens_mg = FArray("r", [(1, o.c_tot)])

    # -- data movement (host fields use the reference's dims ttc with pl ghosts)
    @property
    def pl(self):
        return self.M.v_pl

    def dom(self, ib):
        return self.M.v_dom.g(ib + 1)

    def put_field(self, name, ib, a):
        """a: numpy (ttc_k, ttc_j, ttc_i), x fastest (C order)."""
        arr = getattr(self.dom(ib), "c_" + name)
        arr.d = [float(x) for x in np.asarray(a, dtype=np.float64).ravel(order="C")]

    def get_field(self, name, ib):
        arr = getattr(self.dom(ib), "c_" + name)
        return np.array(arr.d).reshape(arr.ext[2], arr.ext[1], arr.ext[0])

    def cof(self, ib):
        return np.array(self.dom(ib).c_cof.d)

    def level_phi(self, g, ib):
        """Level-g iterate of block ib (canonical (nz+2, ny+2, nx+2), x fastest)."""
        o = self.dom(ib)
        gl = min(g, o.c_ngrid)
        ni = _idiv(o.c_iep - o.c_isp + 1, 2 ** (gl - 1)) + 2
        nj = _idiv(o.c_jep - o.c_jsp + 1, 2 ** (gl - 1)) + 2
        nk = _idiv(o.c_kep - o.c_ksp + 1, 2 ** (gl - 1)) + 2
        base = o.c_faz.g(g) - ni * nj * nk       # mgsolver.for: ijkphi = ... + faz(g) - nijk
        c = np.array(o.c_cof.d[base: base + ni * nj * nk])   # cof(base+1 ...) is d[base ...]
        return c.reshape(nk, ni, nj).transpose(0, 2, 1).copy()

    def set_level_phi(self, g, ib, a):
        o = self.dom(ib)
        gl = min(g, o.c_ngrid)
        ni = _idiv(o.c_iep - o.c_isp + 1, 2 ** (gl - 1)) + 2
        nj = _idiv(o.c_jep - o.c_jsp + 1, 2 ** (gl - 1)) + 2
        nk = _idiv(o.c_kep - o.c_ksp + 1, 2 ** (gl - 1)) + 2
        base = o.c_faz.g(g) - ni * nj * nk
        flat = np.asarray(a, dtype=np.float64).transpose(0, 2, 1).ravel()
        o.c_cof.d[base: base + ni * nj * nk] = [float(x) for x in flat]

    def level_slot(self, g, ib, s):
        """Interior slot s (0..6 coefficients, 7 rhs/residual) of level g, (nz, ny, nx)."""
        o = self.dom(ib)
        gl = min(g, o.c_ngrid)
        ni = _idiv(o.c_iep - o.c_isp + 1, 2 ** (gl - 1)) + 2
        nj = _idiv(o.c_jep - o.c_jsp + 1, 2 ** (gl - 1)) + 2
        nk = _idiv(o.c_kep - o.c_ksp + 1, 2 ** (gl - 1)) + 2
        incr = (ni - 2) * (nj - 2) * (nk - 2)
        base = o.c_faz.g(g) + s * incr           # cof(faz + s*incr + 1 ...)
        c = np.array(o.c_cof.d[base: base + incr])
        return c.reshape(nk - 2, ni - 2, nj - 2).transpose(0, 2, 1).copy()

    def set_level_slot(self, g, ib, s, a):
        o = self.dom(ib)
        gl = min(g, o.c_ngrid)
        ni = _idiv(o.c_iep - o.c_isp + 1, 2 ** (gl - 1)) + 2
        nj = _idiv(o.c_jep - o.c_jsp + 1, 2 ** (gl - 1)) + 2
        nk = _idiv(o.c_kep - o.c_ksp + 1, 2 ** (gl - 1)) + 2
        incr = (ni - 2) * (nj - 2) * (nk - 2)
        base = o.c_faz.g(g) + s * incr
        flat = np.asarray(a, dtype=np.float64).transpose(0, 2, 1).ravel()
        o.c_cof.d[base: base + incr] = [float(x) for x in flat]

    def call(self, name, *args):
        return self.ns[name](*args)

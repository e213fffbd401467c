"""Fortran-77 to C translator used to build the reference oracle.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the ``simson_b200`` package,
its CUDA kernels or its C ABI) imports or links what this file produces.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline arm
touch the oracle, and only as the checker.

Why it exists: the reference (Simson ``bla``) is Fortran 77 and this machine
has no Fortran compiler.  Instead of hand-restating ~6000 lines of the hot path
(and guessing at operation order), ``oracle/build_ref.py`` runs this translator
over the reference's own source files where they lie and compiles the result
with gcc into ``oracle/_ref/`` (git-ignored).  The translation is mechanical and
keeps Fortran semantics:

* every actual argument is passed by address (Fortran call by reference);
* arrays are column-major with their declared (possibly adjustable) bounds;
* ``-fdefault-real-8``: ``real`` is ``double``, ``complex`` is
  ``double _Complex``, ``integer`` and ``logical`` are 32-bit ``int``;
* integer division truncates; ``x**n`` with integer ``n`` uses
  ``__builtin_powi`` (what gfortran emits), real exponents use ``pow``;
* DO loops evaluate their bounds once; ``!$omp parallel do`` becomes
  ``#pragma omp parallel for``; labelled DO loops may share a terminal label.

It handles the subset of Fortran the Simson sources use (no COMMON, no
EQUIVALENCE, no character processing in the translated units).  I/O
statements (WRITE/PRINT/FORMAT) are dropped.  Anything it does not understand
raises ``F77Error`` with the file and line, so a silent mistranslation is not
possible for unsupported syntax.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

__all__ = ["F77Error", "translate"]


class F77Error(Exception):
    pass


# ---------------------------------------------------------------------------
# source preprocessing
# ---------------------------------------------------------------------------

@dataclass
class Line:
    file: str
    lineno: int
    text: str


def cpp(text: str, fname: str, defines: set, includes: dict) -> list:
    """Minimal C-preprocessor pass: #ifdef/#ifndef/#else/#endif and includes.

    ``includes`` maps an include name (``par.f``) to replacement text; both the
    ``#include "x"`` and the Fortran ``include 'x'`` forms are expanded."""
    out = []
    stack = []  # each entry: (active_before, taking_branch, seen_true)
    active = True
    for i, raw in enumerate(text.split("\n"), start=1):
        s = raw.strip()
        if s.startswith("#"):
            d = s[1:].strip()
            m = re.match(r"(ifdef|ifndef)\s+(\w+)", d)
            if m:
                cond = (m.group(2) in defines) == (m.group(1) == "ifdef")
                stack.append((active, cond))
                active = active and cond
                continue
            if d.startswith("else"):
                prev_active, cond = stack[-1]
                stack[-1] = (prev_active, not cond)
                active = prev_active and not cond
                continue
            if d.startswith("endif"):
                active = stack.pop()[0]
                continue
            m = re.match(r'include\s+["<](.+)[">]', d)
            if m:
                if active:
                    out.extend(_include(m.group(1), includes, fname, i))
                continue
            if d.startswith("define") or d.startswith("undef"):
                continue
            raise F77Error(f"{fname}:{i}: unsupported directive {s}")
        if not active:
            continue
        m = re.match(r"\s+include\s+'([^']+)'", raw, re.I)
        if m and raw[:1] not in "cC*!":
            out.extend(_include(m.group(1), includes, fname, i))
            continue
        out.append(Line(fname, i, raw))
    if stack:
        raise F77Error(f"{fname}: unterminated #if")
    return out


def _include(name, includes, fname, lineno):
    if name not in includes:
        if name == "mpif.h":
            return []
        raise F77Error(f"{fname}:{lineno}: unknown include {name}")
    return [Line(name, j, t) for j, t in enumerate(includes[name].split("\n"), 1)]


@dataclass
class Stmt:
    label: int | None
    text: str          # lower-cased outside strings, blanks preserved
    file: str
    lineno: int
    omp: str | None = None   # '!$omp' directive text if this is a directive


def _strip_inline_comment(code: str) -> str:
    q = None
    for k, ch in enumerate(code):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "!":
            return code[:k]
    return code


def _lower_outside_strings(s: str) -> str:
    out, q = [], None
    for ch in s:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        else:
            if ch in "'\"":
                q = ch
            out.append(ch.lower())
    return "".join(out)


def fixed_form(lines: list) -> list:
    stmts: list = []
    for ln in lines:
        raw = ln.text.rstrip("\n")
        if not raw.strip():
            continue
        c0 = raw[:1]
        if c0 in "cC*!":
            low = raw.lower()
            if low.startswith("!$omp") or low.startswith("c$omp"):
                stmts.append(Stmt(None, low[5:].strip(), ln.file, ln.lineno, omp=low[5:].strip()))
            continue
        raw = raw[:72]
        lab = raw[:5].strip()
        cont = len(raw) > 5 and raw[5] not in " 0"
        code = _strip_inline_comment(raw[6:])
        if cont:
            if not stmts or stmts[-1].omp is not None:
                raise F77Error(f"{ln.file}:{ln.lineno}: continuation without statement")
            stmts[-1].text += code
            continue
        if not code.strip() and not lab:
            continue
        stmts.append(Stmt(int(lab) if lab else None, code, ln.file, ln.lineno))
    for s in stmts:
        if s.omp is None:
            s.text = _lower_outside_strings(s.text).strip()
    return stmts


# ---------------------------------------------------------------------------
# expressions
# ---------------------------------------------------------------------------

_DOTOPS = ("eq", "ne", "lt", "le", "gt", "ge", "and", "or", "not", "eqv", "neqv", "true", "false")
_TOKRE = re.compile(r"""
    (?P<ws>\s+)
  | (?P<str>'(?:[^']|'')*'|"[^"]*")
  | (?P<dot>\.(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv|true|false)\.)
  | (?P<num>(?:\d+\.(?!(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv)\.)\d*|\.\d+|\d+)(?:[ed][+-]?\d+)?)
  | (?P<id>[a-z_][a-z0-9_$]*)
  | (?P<op>\*\*|//|==|/=|<=|>=|::|=>|[-+*/(),=:<>%])
""", re.X)


def tokenize(s: str, where: str) -> list:
    # fixed form ignores blanks: '2 .' is the real constant '2.'
    s = re.sub(r"(\d)\s+\.(?=\s*(?:[^a-z\s]|$))", r"\1.", s)
    toks, pos = [], 0
    while pos < len(s):
        m = _TOKRE.match(s, pos)
        if not m:
            raise F77Error(f"{where}: cannot tokenize at {s[pos:pos+20]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        toks.append((kind, m.group(kind)))
    return toks


class ExprParser:
    """Precedence-climbing parser for Fortran expressions."""

    def __init__(self, toks, where):
        self.t = toks
        self.i = 0
        self.where = where

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise F77Error(f"{self.where}: expected {val!r}, got {tok[1]!r}")
        self.i += 1
        return tok

    def at_end(self):
        return self.i >= len(self.t)

    def parse(self):
        return self.eqv()

    def eqv(self):
        a = self.lor()
        while self.peek()[1] in (".eqv.", ".neqv."):
            op = self.take()[1]
            a = ("bin", op, a, self.lor())
        return a

    def lor(self):
        a = self.land()
        while self.peek()[1] == ".or.":
            self.take()
            a = ("bin", ".or.", a, self.land())
        return a

    def land(self):
        a = self.lnot()
        while self.peek()[1] == ".and.":
            self.take()
            a = ("bin", ".and.", a, self.lnot())
        return a

    def lnot(self):
        if self.peek()[1] == ".not.":
            self.take()
            return ("un", ".not.", self.lnot())
        return self.rel()

    _REL = {".eq.": "==", ".ne.": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">=",
            "==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">="}

    def rel(self):
        a = self.concat()
        if self.peek()[1] in self._REL:
            op = self._REL[self.take()[1]]
            a = ("bin", op, a, self.concat())
        return a

    def concat(self):
        a = self.add()
        while self.peek()[1] == "//":
            self.take()
            a = ("bin", "//", a, self.add())
        return a

    def add(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = self.mul()
            a = ("un", op, a)
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = ("bin", op, a, self.mul())
        return a

    def mul(self):
        a = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            a = ("bin", op, a, self.power())
        return a

    def power(self):
        a = self.unary_primary()
        if self.peek()[1] == "**":
            self.take()
            b = self.power()  # right associative
            return ("bin", "**", a, b)
        return a

    def unary_primary(self):
        # gfortran extension: a*-b, a**-b
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            return ("un", op, self.power())
        return self.primary()

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return ("num", val)
        if kind == "str":
            self.take()
            return ("str", val)
        if kind == "dot" and val in (".true.", ".false."):
            self.take()
            return ("lit", val == ".true.")
        if kind == "id":
            self.take()
            if self.peek()[1] == "(":
                self.take()
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.arg())
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return ("ref", val, args)
            return ("name", val)
        if val == "(":
            self.take()
            a = self.parse()
            if self.peek()[1] == ",":  # complex constant (re, im)
                self.take()
                b = self.parse()
                self.take(")")
                return ("cplx", a, b)
            self.take(")")
            return ("paren", a)
        raise F77Error(f"{self.where}: unexpected token {val!r}")

    def arg(self):
        # array section  lo:hi  or  :
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.parse()
            return ("slice", None, hi)
        a = self.parse()
        if self.peek()[1] == ":":
            self.take()
            hi = None if self.peek()[1] in (",", ")") else self.parse()
            return ("slice", a, hi)
        return a


def parse_expr(s: str, where: str):
    p = ExprParser(tokenize(s, where), where)
    e = p.parse()
    if not p.at_end():
        raise F77Error(f"{where}: trailing tokens in expression {s!r}")
    return e


def split_top(s: str, sep=",") -> list:
    """Split at top-level separators (outside parentheses and strings)."""
    parts, depth, q, cur = [], 0, None, []
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur))
    return [p.strip() for p in parts]


def match_paren(s: str, start: int) -> int:
    """Index of the ')' matching the '(' at ``start``."""
    depth, q = 0, None
    for k in range(start, len(s)):
        ch = s[k]
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return k
    raise F77Error(f"unbalanced parentheses in {s!r}")


# ---------------------------------------------------------------------------
# program units
# ---------------------------------------------------------------------------

CTYPE = {"i": "int", "r": "double", "l": "int", "c": "double _Complex", "s": "char"}


@dataclass
class Var:
    name: str
    typ: str | None = None         # i r l c s
    dims: list | None = None       # list of (lo_ast, hi_ast|None for '*')
    dummy: bool = False
    param: object = None           # AST of the value for PARAMETER
    external: bool = False
    data: list | None = None       # list of value ASTs (DATA)
    global_: bool = False
    char: bool = False


@dataclass
class Unit:
    kind: str                      # subroutine function program
    name: str
    args: list
    rtype: str | None = None
    vars: dict = field(default_factory=dict)
    body: list = field(default_factory=list)
    implicit_none: bool = False
    file: str = ""
    param_order: list = field(default_factory=list)

    def var(self, name, create=True):
        v = self.vars.get(name)
        if v is None and create:
            v = self.vars[name] = Var(name)
        return v


_TYPE_RE = re.compile(r"^(integer|real|logical|complex|character|double\s*precision|doubleprecision)"
                      r"(\*\s*\d+|\*\(\s*\*\s*\)|\s*\(\s*(?:len\s*=\s*)?[\w*]+\s*\))?"
                      r"(?=[\s,:]|$)(.*)$")


def _typ_letter(tname: str) -> str:
    tname = tname.replace(" ", "")
    return {"integer": "i", "real": "r", "logical": "l", "complex": "c",
            "character": "s", "doubleprecision": "r"}[tname]


def parse_units(stmts: list) -> list:
    units: list = []
    cur: Unit | None = None
    for st in stmts:
        where = f"{st.file}:{st.lineno}"
        t = st.text
        if st.omp is not None:
            if cur is not None:
                cur.body.append(("omp", st))
            continue
        if cur is None:
            m = re.match(r"^(?:(integer|real|logical|double\s*precision)\s+)?(subroutine|function|program)\s+(\w+)\s*(\(.*\))?\s*$", t)
            if not m:
                if t.startswith("block data"):
                    raise F77Error(f"{where}: block data unsupported")
                raise F77Error(f"{where}: statement outside a program unit: {t!r}")
            args = []
            if m.group(4):
                inner = m.group(4).strip()[1:-1].strip()
                args = [a.strip() for a in inner.split(",")] if inner else []
            cur = Unit(m.group(2), m.group(3), args, file=st.file)
            if m.group(1):
                cur.rtype = _typ_letter(m.group(1))
            for a in args:
                cur.var(a).dummy = True
            continue
        if re.match(r"^end(\s*(subroutine|function|program)(\s+\w+)?)?$", t):
            if st.label is not None:
                cur.body.append(("stmt", Stmt(st.label, "continue", st.file, st.lineno)))
            units.append(cur)
            cur = None
            continue
        if _spec_stmt(cur, st, where):
            continue
        cur.body.append(("stmt", st))
    if cur is not None:
        raise F77Error(f"missing END for unit {cur.name}")
    return units


def _parse_entity_dims(decl: str, where: str):
    """'name(d1,d2)' -> (name, [(lo,hi),...]) ; 'name' -> (name, None)."""
    m = re.match(r"^(\w+)\s*(\((.*)\))?\s*(\*\s*\d+)?$", decl.strip())
    if not m:
        raise F77Error(f"{where}: bad declaration entity {decl!r}")
    name = m.group(1)
    if m.group(2) is None:
        return name, None
    dims = []
    for d in split_top(m.group(3)):
        if d == "*":
            dims.append((("num", "1"), None))
            continue
        parts = split_top(d, ":")
        if len(parts) == 1:
            dims.append((("num", "1"), parse_expr(parts[0], where)))
        elif len(parts) == 2:
            hi = None if parts[1] == "*" else parse_expr(parts[1], where)
            dims.append((parse_expr(parts[0], where), hi))
        else:
            raise F77Error(f"{where}: bad dimension {d!r}")
    return name, dims


def _spec_stmt(u: Unit, st: Stmt, where: str) -> bool:
    t = st.text
    if t == "implicit none":
        u.implicit_none = True
        return True
    if t.startswith("implicit "):
        raise F77Error(f"{where}: only IMPLICIT NONE is supported")
    if re.match(r"^(save|intrinsic)\b", t):
        return True
    m = re.match(r"^external\s+(.*)$", t)
    if m:
        for n in split_top(m.group(1)):
            u.var(n).external = True
        return True
    m = re.match(r"^parameter\s*\((.*)\)$", t)
    if m:
        for item in split_top(m.group(1)):
            n, e = item.split("=", 1)
            v = u.var(n.strip())
            v.param = parse_expr(e.strip(), where)
            u.param_order.append(v.name)
        return True
    m = re.match(r"^dimension\s+(.*)$", t)
    if m:
        for ent in split_top(m.group(1)):
            n, dims = _parse_entity_dims(ent, where)
            u.var(n).dims = dims
        return True
    m = re.match(r"^data\s+(.*)$", t)
    if m:
        body = m.group(1)
        for mm in re.finditer(r"(\w+)\s*/([^/]*)/", body):
            v = u.var(mm.group(1))
            vals = []
            for item in split_top(mm.group(2)):
                if "*" in item and re.match(r"^\d+\s*\*", item):
                    cnt, val = item.split("*", 1)
                    vals.extend([parse_expr(val, where)] * int(cnt))
                else:
                    vals.append(parse_expr(item, where))
            v.data = vals
        return True
    m = _TYPE_RE.match(t)
    if m and not re.match(r"^(real|integer|logical|complex)\s*function\b", t):
        tl = _typ_letter(m.group(1))
        rest = m.group(3).strip()
        attrs = []
        if "::" in rest:
            a, rest = rest.split("::", 1)
            attrs = [x.strip() for x in split_top(a.strip().lstrip(","))] if a.strip() else []
            rest = rest.strip()
        elif rest.startswith(","):
            raise F77Error(f"{where}: attribute list without '::'")
        is_param = "parameter" in attrs
        is_ext = "external" in attrs
        for ent in split_top(rest):
            init = None
            if "=" in ent and not ent.startswith("("):
                ent, init = ent.split("=", 1)
            name, dims = _parse_entity_dims(ent, where)
            v = u.var(name)
            v.typ = tl
            if tl == "s":
                v.char = True
            if dims is not None:
                v.dims = dims
            if is_ext:
                v.external = True
            if init is not None:
                if is_param:
                    v.param = parse_expr(init.strip(), where)
                    u.param_order.append(name)
                elif tl != "s":
                    v.data = [parse_expr(init.strip(), where)]
        return True
    return False


# ---------------------------------------------------------------------------
# C code generation
# ---------------------------------------------------------------------------

INTRINSIC_R = {"sqrt", "exp", "log", "log10", "sin", "cos", "tan", "asin", "acos", "atan",
               "atan2", "sinh", "cosh", "tanh"}
INTRINSICS = INTRINSIC_R | {"abs", "min", "max", "mod", "modulo", "sign", "real", "float", "dble",
                            "int", "nint", "aint", "anint", "aimag", "conjg", "cmplx", "dcmplx",
                            "omp_get_thread_num", "omp_get_num_threads", "floor", "ceiling", "iabs",
                            "amax1", "amin1", "min0", "max0", "dabs", "dsqrt", "idint", "ifix",
                            "epsilon", "huge", "dmax1", "dmin1", "dcos", "dsin"}


class Ctx:
    def __init__(self, unit: Unit, gen: "Translator"):
        self.u = unit
        self.g = gen
        self.tmp = 0

    def where(self, st):
        return f"{st.file}:{st.lineno}"

    def vtype(self, name) -> str:
        v = self.u.vars.get(name)
        if v is None or v.typ is None:
            if v is not None and v.param is not None:
                return self.etype(v.param)
            gv = self.g.globals.get(name)
            if gv is not None and gv.typ is not None:
                return gv.typ
            if self.u.implicit_none and not (v is not None and v.dummy):
                raise F77Error(f"{self.u.file}: unit {self.u.name}: undeclared {name}")
            return "i" if name[0] in "ijklmn" else "r"
        return v.typ

    def lookup(self, name) -> Var | None:
        v = self.u.vars.get(name)
        if v is not None:
            return v
        return self.g.globals.get(name)

    # --- types -------------------------------------------------------------
    def etype(self, e) -> str:
        k = e[0]
        if k == "num":
            return "r" if re.search(r"[.ed]", e[1]) else "i"
        if k == "lit":
            return "l"
        if k == "str":
            return "s"
        if k == "cplx":
            return "c"
        if k == "paren":
            return self.etype(e[1])
        if k == "name":
            return self.vtype(e[1])
        if k == "un":
            return "l" if e[1] == ".not." else self.etype(e[2])
        if k == "bin":
            op = e[1]
            if op in ("==", "!=", "<", "<=", ">", ">=", ".and.", ".or.", ".eqv.", ".neqv."):
                return "l"
            a, b = self.etype(e[2]), self.etype(e[3])
            if op == "**" and b == "i":
                return a
            return _promote(a, b)
        if k == "ref":
            name, args = e[1], e[2]
            v = self.lookup(name)
            if v is not None and v.dims is not None:
                return self.vtype(name)
            if v is not None and (v.external or (v.typ is not None and not v.dims)) and name not in INTRINSICS:
                return self.vtype(name)
            return self.intrinsic_type(name, args)
        raise F77Error(f"etype: {e}")

    def intrinsic_type(self, name, args):
        if name in INTRINSIC_R or name in ("dsqrt", "dcos", "dsin"):
            return "c" if self.etype(args[0]) == "c" else "r"
        if name in ("real", "float", "dble", "aimag", "aint", "anint", "amax1", "amin1", "dmax1", "dmin1", "dabs",
                    "epsilon", "huge"):
            if name == "real" and False:
                pass
            return "r"
        if name in ("int", "nint", "idint", "ifix", "floor", "ceiling", "iabs", "min0", "max0",
                    "omp_get_thread_num", "omp_get_num_threads"):
            return "i"
        if name in ("conjg", "cmplx", "dcmplx"):
            return "c"
        if name in ("abs",):
            t = self.etype(args[0])
            return "r" if t == "c" else t
        if name in ("min", "max", "mod", "modulo", "sign"):
            t = self.etype(args[0])
            for a in args[1:]:
                t = _promote(t, self.etype(a))
            return t
        f = self.g.functions.get(name)
        if f is not None:
            return f.rtype or ("i" if name[0] in "ijklmn" else "r")
        raise F77Error(f"unit {self.u.name}: unknown function {name}")

    # --- expressions -------------------------------------------------------
    def cname(self, name):
        return "v_" + name

    def scalar_ref(self, name) -> str:
        v = self.lookup(name)
        if v is not None and v.param is not None and not v.dummy:
            return self.cname(name)
        if v is not None and v.dummy and (v.dims is None):
            return f"(*{self.cname(name)})"
        return self.cname(name)

    def index(self, name, args, st) -> str:
        v = self.lookup(name)
        n = len(v.dims)
        if len(args) != n:
            raise F77Error(f"{self.where(st)}: {name} has rank {n}, indexed with {len(args)}")
        cn = self.cname(name)
        terms = None
        for k in range(n - 1, -1, -1):
            ik = f"((long)({self.expr(args[k], st)})-{cn}__l{k})"
            if terms is None:
                terms = ik
            else:
                terms = f"{ik}+{cn}__e{k}*({terms})"
        return f"{cn}[{terms}]"

    def expr(self, e, st) -> str:
        k = e[0]
        if k == "cexpr":  # a C expression made by the translator itself
            return e[1]
        if k == "num":
            s = e[1].replace("d", "e")
            return s
        if k == "lit":
            return "1" if e[1] else "0"
        if k == "str":
            raise F77Error(f"{self.where(st)}: string expression unsupported")
        if k == "cplx":
            return f"((double)({self.expr(e[1], st)})+(double)({self.expr(e[2], st)})*_Complex_I)"
        if k == "paren":
            return f"({self.expr(e[1], st)})"
        if k == "name":
            v = self.lookup(e[1])
            if v is not None and v.dims is not None:
                raise F77Error(f"{self.where(st)}: whole array {e[1]} in expression")
            return self.scalar_ref(e[1])
        if k == "un":
            if e[1] == ".not.":
                return f"(!{self.expr(e[2], st)})"
            return f"({e[1]}{self.expr(e[2], st)})"
        if k == "bin":
            op = e[1]
            a, b = self.expr(e[2], st), self.expr(e[3], st)
            if op == "**":
                ta, tb = self.etype(e[2]), self.etype(e[3])
                if tb == "i":
                    if ta == "i":
                        return f"f77_ipow({a},{b})"
                    if ta == "r":
                        return f"__builtin_powi({a},{b})"
                    return f"cpow({a},(double)({b}))"
                if ta == "c" or tb == "c":
                    return f"cpow({a},{b})"
                return f"pow({a},{b})"
            if op == ".and.":
                return f"({a}&&{b})"
            if op == ".or.":
                return f"({a}||{b})"
            if op == ".eqv.":
                return f"((!!{a})==(!!{b}))"
            if op == ".neqv.":
                return f"((!!{a})!=(!!{b}))"
            if op == "//":
                raise F77Error(f"{self.where(st)}: concatenation unsupported")
            return f"({a}{op}{b})"
        if k == "ref":
            name, args = e[1], e[2]
            v = self.lookup(name)
            if v is not None and v.dims is not None:
                if any(a[0] == "slice" for a in args):
                    raise F77Error(f"{self.where(st)}: array section in expression")
                return self.index(name, args, st)
            if name in INTRINSICS and not (v is not None and v.external):
                return self.intrinsic(name, args, st)
            return self.fcall(name, args, st)
        if k == "slice":
            raise F77Error(f"{self.where(st)}: array section unsupported")
        raise F77Error(f"expr: {e}")

    def intrinsic(self, name, args, st) -> str:
        xs = [self.expr(a, st) for a in args]
        ts = [self.etype(a) for a in args]
        name = {"dabs": "abs", "iabs": "abs", "dsqrt": "sqrt", "dcos": "cos", "dsin": "sin",
                "amax1": "max", "amin1": "min", "dmax1": "max", "dmin1": "min", "max0": "max",
                "min0": "min", "idint": "int", "ifix": "int", "dcmplx": "cmplx"}.get(name, name)
        if name in INTRINSIC_R:
            if ts[0] == "c":
                return f"c{name}({', '.join(xs)})"
            return f"{name}({', '.join('(double)(' + x + ')' for x in xs)})"
        if name == "abs":
            return {"i": f"abs({xs[0]})", "r": f"fabs({xs[0]})", "c": f"cabs({xs[0]})"}[ts[0]]
        if name in ("min", "max"):
            t = ts[0]
            for tt in ts[1:]:
                t = _promote(t, tt)
            fn = f"f77_{name}{'i' if t == 'i' else 'd'}"
            acc = xs[0]
            for x in xs[1:]:
                acc = f"{fn}({acc},{x})"
            return acc
        if name == "mod":
            t = _promote(ts[0], ts[1])
            return f"({xs[0]}%{xs[1]})" if t == "i" else f"fmod({xs[0]},{xs[1]})"
        if name == "modulo":
            t = _promote(ts[0], ts[1])
            return f"f77_moduloi({xs[0]},{xs[1]})" if t == "i" else f"f77_modulod({xs[0]},{xs[1]})"
        if name == "sign":
            t = _promote(ts[0], ts[1])
            return f"f77_signi({xs[0]},{xs[1]})" if t == "i" else f"copysign(fabs((double)({xs[0]})),(double)({xs[1]}))"
        if name in ("real", "float", "dble"):
            return f"creal({xs[0]})" if ts[0] == "c" else f"((double)({xs[0]}))"
        if name == "int":
            return f"((int)({xs[0]}))"
        if name == "nint":
            return f"((int)lround({xs[0]}))"
        if name == "aint":
            return f"trunc({xs[0]})"
        if name == "anint":
            return f"round({xs[0]})"
        if name == "floor":
            return f"((int)floor({xs[0]}))"
        if name == "ceiling":
            return f"((int)ceil({xs[0]}))"
        if name == "aimag":
            return f"cimag({xs[0]})"
        if name == "conjg":
            return f"conj({xs[0]})"
        if name == "cmplx":
            im = xs[1] if len(xs) > 1 else "0.0"
            return f"((double)({xs[0]})+(double)({im})*_Complex_I)"
        if name == "omp_get_thread_num":
            return "f77_omp_thread()"
        if name == "omp_get_num_threads":
            return "f77_omp_nthreads()"
        if name == "epsilon":
            return "DBL_EPSILON"
        if name == "huge":
            return "DBL_MAX" if ts[0] == "r" else "INT_MAX"
        raise F77Error(f"{self.where(st)}: intrinsic {name}")

    def actual(self, a, st, dummy_type=None) -> str:
        """An actual argument: always an address (call by reference)."""
        if a[0] == "name":
            v = self.lookup(a[1])
            if v is not None and v.dims is not None:
                return self.cname(a[1])
            if v is not None and v.param is not None and not v.dummy:
                t = dummy_type or self.etype(a)
                return f"&({CTYPE[t]}){{{self.cname(a[1])}}}"
            if v is not None and v.dummy:
                return self.cname(a[1])
            if v is not None and v.char:
                # program-level character variables (file names) are not
                # declared: no translated unit processes characters, so they
                # pass as null, like character literals
                return "(char*)0"
            if v is not None and (v.external or a[1] in self.g.functions) and v.typ is None:
                return f"(void*)f_{a[1]}"
            return f"&{self.cname(a[1])}"
        if a[0] == "ref":
            v = self.lookup(a[1])
            if v is not None and v.dims is not None:
                return "&" + self.index(a[1], a[2], st)
        if a[0] == "str":
            return "(void*)0"
        t = dummy_type or self.etype(a)
        return f"&({CTYPE[t]}){{{self.expr(a, st)}}}"

    def fcall(self, name, args, st) -> str:
        self.g.called.add(name)
        self.g.fcalled[name] = self.etype(("ref", name, args))
        xs = [self.actual(a, st) for a in args]
        return f"f_{name}({', '.join(xs)})"


def _promote(a, b):
    order = {"l": 0, "i": 1, "r": 2, "c": 3, "s": -1}
    return a if order[a] >= order[b] else b


class Translator:
    def __init__(self):
        self.units: list = []
        self.functions: dict = {}
        self.subroutines: dict = {}
        self.globals: dict = {}          # program-level variables (main unit)
        self.called: set = set()
        self.fcalled: dict = {}
        self.global_params: dict = {}    # from par.f (emitted once)
        self.par_names: set = set()

    def add(self, units):
        for u in units:
            if u.kind == "function":
                self.functions[u.name] = u
            elif u.kind == "subroutine":
                self.subroutines[u.name] = u
            self.units.append(u)

    # --- declarations ------------------------------------------------------
    def param_is_const_int(self, ctx, e) -> bool:
        k = e[0]
        if k == "num":
            return not re.search(r"[.ed]", e[1])
        if k == "name":
            v = ctx.lookup(e[1])
            return v is not None and v.param is not None and self.param_is_const_int(ctx, v.param)
        if k == "paren":
            return self.param_is_const_int(ctx, e[1])
        if k == "un":
            return e[1] in "+-" and self.param_is_const_int(ctx, e[2])
        if k == "bin":
            return e[1] in "+-*/" and self.param_is_const_int(ctx, e[2]) and self.param_is_const_int(ctx, e[3])
        return False

    def emit_params(self, ctx, names, indent, skip=()) -> list:
        out = []
        for n in names:
            if n in skip:
                continue
            v = ctx.lookup(n)
            t = ctx.vtype(n)
            if t == "s":
                continue
            cval = None
            if t == "i":
                try:
                    cval = self.const_eval(ctx, v.param)
                except F77Error:
                    cval = None
            if cval is not None:
                out.append(f"{indent}enum {{ v_{n} = {cval} }};")
            elif t == "i" and self.param_is_const_int(ctx, v.param):
                out.append(f"{indent}enum {{ v_{n} = {ctx.expr(v.param, None)} }};")
            else:
                out.append(f"{indent}const {CTYPE[t]} v_{n} = {ctx.expr(v.param, None)};")
        return out

    def dims_code(self, ctx, name, v, indent) -> list:
        out = []
        for k, (lo, hi) in enumerate(v.dims):
            lo_s = ctx.expr(lo, None)
            out.append(f"{indent}const long v_{name}__l{k} = (long)({lo_s});")
            if hi is None:
                out.append(f"{indent}const long v_{name}__e{k} = 1; (void)v_{name}__e{k};")
            else:
                out.append(f"{indent}const long v_{name}__e{k} = (long)({ctx.expr(hi, None)})-v_{name}__l{k}+1;")
            out.append(f"{indent}(void)v_{name}__l{k};")
        return out

    def array_size_expr(self, ctx, v) -> str:
        parts = []
        for lo, hi in v.dims:
            if hi is None:
                raise F77Error(f"assumed-size array {v.name} cannot be allocated")
            parts.append(f"((long)({ctx.expr(hi, None)})-(long)({ctx.expr(lo, None)})+1)")
        return "*".join(parts)

    def const_size(self, ctx, v) -> int:
        """Element count if every bound is a constant expression, else 0."""
        n = 1
        for lo, hi in v.dims:
            if hi is None:
                return 0
            try:
                a = self.const_eval(ctx, lo)
                b = self.const_eval(ctx, hi)
            except F77Error:
                return 0
            n *= max(0, b - a + 1)
        return n

    def const_eval(self, ctx, e) -> int:
        k = e[0]
        if k == "num" and not re.search(r"[.ed]", e[1]):
            return int(e[1])
        if k == "name":
            v = ctx.lookup(e[1])
            if v is not None and v.param is not None:
                return self.const_eval(ctx, v.param)
        if k == "paren":
            return self.const_eval(ctx, e[1])
        if k == "un" and e[1] in "+-":
            x = self.const_eval(ctx, e[2])
            return -x if e[1] == "-" else x
        if k == "ref" and e[1] in ("min", "max", "mod") and ctx.lookup(e[1]) is None:
            xs = [self.const_eval(ctx, a) for a in e[2]]
            if e[1] == "min":
                return min(xs)
            if e[1] == "max":
                return max(xs)
            r = abs(xs[0]) % abs(xs[1])
            return r if xs[0] >= 0 else -r
        if k == "bin" and e[1] in "+-*/":
            a, b = self.const_eval(ctx, e[2]), self.const_eval(ctx, e[3])
            if e[1] == "+":
                return a + b
            if e[1] == "-":
                return a - b
            if e[1] == "*":
                return a * b
            q = abs(a) // abs(b)
            return q if (a >= 0) == (b >= 0) else -q
        raise F77Error("not constant")

    def signature(self, u: Unit) -> str:
        ctx = Ctx(u, self)
        ps = []
        for a in u.args:
            v = u.vars[a]
            if a in self.functions or (v.external and v.typ is None):
                ps.append(f"void *v_{a}")
                continue
            t = ctx.vtype(a)
            if t == "s":
                ps.append(f"char *v_{a}")
            else:
                ps.append(f"{CTYPE[t]} *v_{a}")
        ret = "void" if u.kind == "subroutine" else CTYPE[u.rtype or ("i" if u.name[0] in "ijklmn" else "r")]
        return f"{ret} f_{u.name}({', '.join(ps) if ps else 'void'})"

    # --- statements --------------------------------------------------------
    def gen_body(self, ctx: Ctx, body: list, indent="  ") -> list:
        out: list = []
        stack: list = []
        targets = set()
        for kind, st in body:
            if kind == "stmt":
                m = re.match(r"^go\s*to\s*(\d+)$", st.text)
                if m:
                    targets.add(int(m.group(1)))
                m = re.match(r"^if\s*\(.*\)\s*go\s*to\s*(\d+)$", st.text)
                if m:
                    targets.add(int(m.group(1)))
        pending_omp = None

        def ind():
            return indent + "  " * len(stack)

        for kind, st in body:
            if kind == "omp":
                d = st.omp
                m = re.match(r"^parallel\s+do\b(.*)$", d)
                if m:
                    clauses = m.group(1)
                    clauses = re.sub(r"\b(private|shared|firstprivate|lastprivate)\s*\(([^)]*)\)",
                                     lambda mm: f"{mm.group(1)}({', '.join('v_' + x.strip() for x in mm.group(2).split(','))})",
                                     clauses)
                    pending_omp = f"#pragma omp parallel for {clauses.strip()}"
                continue
            where = ctx.where(st)
            t = st.text
            if st.label is not None and st.label in targets:
                out.append(f"{ind()}L{st.label}:;")
            # block constructs
            m = re.match(r"^if\s*\((.*)\)\s*then$", t)
            if m and _balanced_if(t):
                out.append(f"{ind()}if ({ctx.expr(parse_expr(m.group(1), where), st)}) {{")
                stack.append(("if", None))
                self._close_do(st, stack, out, ind)
                continue
            m = re.match(r"^else\s*if\s*\((.*)\)\s*then$", t)
            if m:
                stack.pop()
                out.append(f"{ind()}}} else if ({ctx.expr(parse_expr(m.group(1), where), st)}) {{")
                stack.append(("if", None))
                continue
            if t == "else":
                stack.pop()
                out.append(f"{ind()}}} else {{")
                stack.append(("if", None))
                continue
            if re.match(r"^end\s*if$", t):
                if not stack or stack[-1][0] != "if":
                    raise F77Error(f"{where}: END IF without IF")
                stack.pop()
                out.append(f"{ind()}}}")
                self._close_do(st, stack, out, ind)
                continue
            m = re.match(r"^do\s*(\d+)?\s*,?\s*(\w+)\s*=\s*(.*)$", t)
            if m and len(split_top(m.group(3))) not in (2, 3):
                m = None
            if m and not t.startswith("do while"):
                lab = int(m.group(1)) if m.group(1) else None
                var = m.group(2)
                bounds = split_top(m.group(3))
                if len(bounds) not in (2, 3):
                    raise F77Error(f"{where}: bad DO bounds")
                lo = ctx.expr(parse_expr(bounds[0], where), st)
                hi = ctx.expr(parse_expr(bounds[1], where), st)
                step = ctx.expr(parse_expr(bounds[2], where), st) if len(bounds) == 3 else "1"
                vt = ctx.vtype(var)
                if vt != "i":
                    raise F77Error(f"{where}: non-integer DO variable")
                lv = ctx.scalar_ref(var)
                ctx.tmp += 1
                hn, sn = f"_hi{ctx.tmp}", f"_st{ctx.tmp}"
                out.append(f"{ind()}{{ const int {hn} = {hi}; const int {sn} = {step}; (void){sn};")
                if pending_omp:
                    if step != "1":
                        raise F77Error(f"{where}: omp loop with step")
                    out.append(pending_omp)
                    pending_omp = None
                    out.append(f"{ind()}for ({lv} = {lo}; {lv} <= {hn}; {lv}++) {{")
                elif re.fullmatch(r"-?\d+", step):
                    cmp = "<=" if int(step) > 0 else ">="
                    out.append(f"{ind()}for ({lv} = {lo}; {lv} {cmp} {hn}; {lv} += {sn}) {{")
                else:
                    out.append(f"{ind()}for ({lv} = {lo}; ({sn} > 0) ? ({lv} <= {hn}) : ({lv} >= {hn}); {lv} += {sn}) {{")
                stack.append(("do", lab))
                continue
            if re.match(r"^end\s*do$", t):
                if not stack or stack[-1] != ("do", None):
                    raise F77Error(f"{where}: END DO mismatch")
                stack.pop()
                out.append(f"{ind()}}} }}")
                self._close_do(st, stack, out, ind)
                continue
            # simple statements
            line = self.simple(ctx, st, t, where)
            if line is not None:
                out.append(f"{ind()}{line}")
            self._close_do(st, stack, out, ind)
        if stack:
            raise F77Error(f"unit {ctx.u.name}: unclosed block {stack[-1]}")
        return out

    def _close_do(self, st, stack, out, ind):
        if st.label is None:
            return
        while stack and stack[-1] == ("do", st.label):
            stack.pop()
            out.append(f"{ind()}}} }}")

    def simple(self, ctx: Ctx, st, t, where):
        if t == "continue":
            return ";"
        m = re.match(r"^go\s*to\s*(\d+)$", t)
        if m:
            return f"goto L{m.group(1)};"
        if t == "return":
            if ctx.u.kind == "function":
                return f"return v_{ctx.u.name};"
            return "return;"
        m = re.match(r"^stop\b\s*(.*)$", t)
        if m:
            code = m.group(1).strip()
            if not re.fullmatch(r"\d*", code):
                code = "1"
            return f"f77_stop({code or '0'});"
        if re.match(r"^(write|print|format|open|close|rewind|flush|inquire|backspace|endfile)\b", t):
            return None
        if re.match(r"^read\b", t):
            raise F77Error(f"{where}: READ unsupported")
        m = re.match(r"^if\s*\(", t)
        if m and not t.endswith("then") or (m and not _balanced_if(t)):
            k = match_paren(t, t.index("("))
            cond = ctx.expr(parse_expr(t[t.index("(") + 1:k], where), st)
            rest = t[k + 1:].strip()
            inner = self.simple(ctx, st, rest, where)
            return f"if ({cond}) {{ {inner or ';'} }}"
        m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", t)
        if m:
            name = m.group(1)
            self.called.add(name)
            args = []
            if m.group(2):
                inner = m.group(3).strip()
                if inner:
                    p = ExprParser(tokenize(inner, where), where)
                    while True:
                        args.append(p.parse())
                        if p.peek()[1] == ",":
                            p.take()
                            continue
                        break
                    if not p.at_end():
                        raise F77Error(f"{where}: bad call arguments")
            callee = self.subroutines.get(name)
            dtypes = [None] * len(args)
            if callee is not None:
                cctx = Ctx(callee, self)
                if len(callee.args) != len(args):
                    raise F77Error(f"{where}: call {name} with {len(args)} args, expects {len(callee.args)}")
                for k, an in enumerate(callee.args):
                    cv = callee.vars[an]
                    if not (cv.external and cv.typ is None):
                        dtypes[k] = cctx.vtype(an)
            xs = [ctx.actual(a, st, dtypes[k]) for k, a in enumerate(args)]
            return f"f_{name}({', '.join(xs)});"
        # assignment
        eq = _find_assign(t)
        if eq is None:
            raise F77Error(f"{where}: unsupported statement {t!r}")
        lhs_s, rhs_s = t[:eq].strip(), t[eq + 1:].strip()
        lhs = parse_expr(lhs_s, where)
        rhs = parse_expr(rhs_s, where)
        if lhs[0] == "name":
            v = ctx.lookup(lhs[1])
            if v is not None and v.dims is not None:
                # whole-array assignment of a scalar
                if ctx.etype(rhs) in ("i", "r", "l", "c") and not (rhs[0] == "name" and ctx.lookup(rhs[1]) and ctx.lookup(rhs[1]).dims):
                    size = "*".join(f"v_{lhs[1]}__e{k}" for k in range(len(v.dims)))
                    ctx.tmp += 1
                    return f"for (long _w{ctx.tmp} = 0; _w{ctx.tmp} < {size}; _w{ctx.tmp}++) v_{lhs[1]}[_w{ctx.tmp}] = {ctx.expr(rhs, st)};"
                raise F77Error(f"{where}: array assignment unsupported")
            if lhs[1] == ctx.u.name and ctx.u.kind == "function":
                return f"v_{lhs[1]} = {ctx.expr(rhs, st)};"
            return f"{ctx.scalar_ref(lhs[1])} = {ctx.expr(rhs, st)};"
        if lhs[0] == "ref":
            v = ctx.lookup(lhs[1])
            if v is None or v.dims is None:
                raise F77Error(f"{where}: assignment to non-array {lhs[1]}(...)")
            if any(a[0] == "slice" for a in lhs[2]):
                # scalar assigned to a section with explicit bounds: a loop nest
                if any(a[0] == "slice" and (a[1] is None or a[2] is None) for a in lhs[2]) or \
                        ctx.etype(rhs) not in ("i", "r", "l", "c"):
                    raise F77Error(f"{where}: array-section assignment unsupported")
                idx, loops = [], []
                for a in lhs[2]:
                    if a[0] == "slice":
                        ctx.tmp += 1
                        iv = f"_s{ctx.tmp}"
                        loops.append(f"for (long {iv} = {ctx.expr(a[1], st)}; {iv} <= {ctx.expr(a[2], st)}; {iv}++)")
                        idx.append(("cexpr", iv))
                    else:
                        idx.append(a)
                return " ".join(loops) + f" {ctx.index(lhs[1], idx, st)} = {ctx.expr(rhs, st)};"
            return f"{ctx.index(lhs[1], lhs[2], st)} = {ctx.expr(rhs, st)};"
        raise F77Error(f"{where}: bad assignment target")

    # --- units -------------------------------------------------------------
    def gen_unit(self, u: Unit) -> list:
        ctx = Ctx(u, self)
        out = [self.signature(u) + " {"]
        ind = "  "
        out += self.emit_params(ctx, u.param_order, ind, skip=self.par_names)
        # locals
        for n, v in u.vars.items():
            if v.dummy or v.param is not None or v.char:
                continue
            if v.external and v.typ is None:
                continue
            if n in self.functions and v.dims is None and n != u.name:
                continue
            if v.external:
                continue
            t = CTYPE[ctx.vtype(n)]
            if v.dims is None:
                if v.data:
                    out.append(f"{ind}static {t} v_{n} = {ctx.expr(v.data[0], None)};")
                else:
                    out.append(f"{ind}{t} v_{n}; (void)v_{n};")
        for n, v in u.vars.items():
            if v.dims is None or v.char or v.param is not None:
                continue
            out += self.dims_code(ctx, n, v, ind)
            if not v.dummy:
                t = CTYPE[ctx.vtype(n)]
                size = self.array_size_expr(ctx, v)
                if v.data:
                    vals = ", ".join(ctx.expr(x, None) for x in v.data)
                    out.append(f"{ind}static {t} v_{n}[{size}] = {{{vals}}};")
                elif self.const_size(ctx, v) > 4096:
                    out.append(f"{ind}static __thread {t} v_{n}[{size}];")
                else:
                    out.append(f"{ind}{t} v_{n}[{size}];")
        out += self.gen_body(ctx, u.body, ind)
        if u.kind == "function":
            out.append(f"{ind}return v_{u.name};")
        out.append("}")
        return out


def _balanced_if(t: str) -> bool:
    """True if 'if (...) then' really is a block IF (the paren closes before 'then')."""
    k = match_paren(t, t.index("("))
    return t[k + 1:].strip() == "then"


def _find_assign(t: str):
    depth, q = 0, None
    for k, ch in enumerate(t):
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            nxt = t[k + 1:k + 2]
            prv = t[k - 1:k] if k else ""
            if nxt != "=" and prv not in "<>/=":
                return k
    return None


RUNTIME = r"""
#include <math.h>
#include <complex.h>
#include <float.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
static inline int f77_omp_thread(void) { return omp_get_thread_num(); }
static inline int f77_omp_nthreads(void) { return omp_get_num_threads(); }
#else
static inline int f77_omp_thread(void) { return 0; }
static inline int f77_omp_nthreads(void) { return 1; }
#endif
static inline int f77_ipow(int b, int e) { int r = 1; if (e < 0) return (b == 1) ? 1 : (b == -1 ? ((e & 1) ? -1 : 1) : 0); while (e) { if (e & 1) r *= b; b *= b; e >>= 1; } return r; }
static inline int f77_maxi(int a, int b) { return a > b ? a : b; }
static inline int f77_mini(int a, int b) { return a < b ? a : b; }
static inline double f77_maxd(double a, double b) { return a > b ? a : b; }
static inline double f77_mind(double a, double b) { return a < b ? a : b; }
static inline int f77_moduloi(int a, int b) { int r = a % b; return (r != 0 && ((r < 0) != (b < 0))) ? r + b : r; }
static inline double f77_modulod(double a, double b) { return a - floor(a / b) * b; }
static inline int f77_signi(int a, int b) { int x = a < 0 ? -a : a; return b >= 0 ? x : -x; }
void f77_stop(int code);
"""


def translate(sources: list, par_text: str, defines=frozenset(), main_ranges=None,
              stubs_noop=(), skip_units=(), provided=()) -> str:
    """Translate Fortran files into one C translation unit.

    sources:     list of (filename, text)
    par_text:    text substituted for ``par.f``
    main_ranges: for a PROGRAM unit, emit only these executable-statement
                 line ranges, each as ``void name(void)``: [(name, lo, hi), ...].
                 The program's variables become file-scope globals and
                 ``f77_main_alloc()`` allocates its arrays (zero-filled).
    stubs_noop:  external subroutines emitted as empty functions (timers).
    """
    tr = Translator()
    includes = {"par.f": par_text}
    # par.f parameters are shared by every unit: emit them once
    par_stmts = fixed_form(cpp(par_text, "par.f", set(defines), {}))
    par_unit = Unit("par", "par", [])
    for st in par_stmts:
        if not _spec_stmt(par_unit, st, f"par.f:{st.lineno}"):
            raise F77Error(f"par.f:{st.lineno}: non-declaration {st.text!r}")
    tr.par_names = set(par_unit.param_order)
    for n in par_unit.param_order:
        tr.globals[n] = par_unit.vars[n]

    all_units = []
    for fname, text in sources:
        stmts = fixed_form(cpp(text, fname, set(defines), includes))
        units = parse_units(stmts)
        all_units += [u for u in units if u.name not in skip_units]
    for u in all_units:
        if u.kind == "function":
            rv = u.vars.get(u.name)
            if u.rtype is None and rv is not None and rv.typ is not None:
                u.rtype = rv.typ
            if u.rtype is None:
                u.rtype = "i" if u.name[0] in "ijklmn" else "r"
            u.var(u.name).typ = u.rtype
    tr.add(all_units)

    out = [RUNTIME]
    pctx = Ctx(par_unit, tr)
    out += tr.emit_params(pctx, par_unit.param_order, "")
    out.append("")
    # prototypes
    protos = []
    for u in tr.units:
        if u.kind in ("subroutine", "function"):
            protos.append(tr.signature(u) + ";")
    out += protos
    main = [u for u in tr.units if u.kind == "program"]
    body = []
    for u in tr.units:
        if u.kind == "program":
            continue
        body += tr.gen_unit(u)
        body.append("")
    if main:
        body += gen_main(tr, main[0], main_ranges or [])
    # stubs for external references that were not translated
    defined = {u.name for u in tr.units}
    stubs = []
    for n in sorted(tr.called - defined):
        if n in INTRINSICS:
            continue
        if n in provided:
            stubs.append(f"void f_{n}();")
            continue
        if n in tr.fcalled:
            t = CTYPE[tr.fcalled[n]]
            stubs.append(f"{t} f_{n}() {{ fprintf(stderr, \"oracle: untranslated function {n} called\\n\"); abort(); return 0; }}")
            continue
        if n in stubs_noop:
            stubs.append(f"void f_{n}() {{ }}")
        else:
            stubs.append(f"void f_{n}() {{ fprintf(stderr, \"oracle: untranslated routine {n} called\\n\"); abort(); }}")
    out += stubs
    out += body
    return "\n".join(out) + "\n"


def gen_main(tr: Translator, u: Unit, ranges: list) -> list:
    """Program unit: globals + allocation + selected executable ranges."""
    ctx = Ctx(u, tr)
    out = []
    for n, v in u.vars.items():
        v.global_ = True
        tr.globals[n] = v
    out += tr.emit_params(ctx, u.param_order, "", skip=tr.par_names)
    decl_arrays = []
    for n, v in u.vars.items():
        if v.param is not None or v.char or v.external:
            continue
        if n in tr.functions or n in tr.subroutines:
            continue
        t = CTYPE[ctx.vtype(n)]
        if v.dims is None:
            out.append(f"{t} v_{n};")
        else:
            out.append(f"{t} *v_{n};")
            for k in range(len(v.dims)):
                out.append(f"long v_{n}__l{k}, v_{n}__e{k};")
            decl_arrays.append(n)
    out.append("void f77_main_alloc(void) {")
    for n in decl_arrays:
        v = u.vars[n]
        for k, (lo, hi) in enumerate(v.dims):
            out.append(f"  v_{n}__l{k} = (long)({ctx.expr(lo, None)});")
            out.append(f"  v_{n}__e{k} = (long)({ctx.expr(hi, None)}) - v_{n}__l{k} + 1;")
        size = "*".join(f"v_{n}__e{k}" for k in range(len(v.dims)))
        t = CTYPE[ctx.vtype(n)]
        out.append(f"  v_{n} = ({t}*)calloc((size_t)({size} > 0 ? {size} : 1), sizeof({t}));")
        out.append(f"  if (!v_{n}) {{ fprintf(stderr, \"oracle: out of memory for {n}\\n\"); abort(); }}")
    out.append("}")
    out.append("void f77_main_free(void) {")
    for n in decl_arrays:
        out.append(f"  free(v_{n}); v_{n} = 0;")
    out.append("}")
    for name, lo, hi in ranges:
        sel = [(k, st) for (k, st) in u.body if lo <= st.lineno <= hi]
        if not sel:
            raise F77Error(f"range {name} {lo}-{hi} selects nothing")
        out.append(f"void {name}(void) {{")
        out += tr.gen_body(ctx, sel, "  ")
        out.append("}")
    return out

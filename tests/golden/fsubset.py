"""A small interpreter for the Fortran 90 subset of BSAM's hot-path leaf
routines, used only to generate golden fixtures (tests/golden/*.npz) from the
reference's own source text.

No Fortran compiler exists in this image, so the reference cannot be built.
Its hot-path routines are plain array statements, DO loops, IF / SELECT CASE,
elemental functions and nodeinfo component references: the leaf routines
(RelaxGrid2D/3D, Operator2D/3D with ULap/UDiv/ULapMob, Source2D/3D,
Restriction2D/3D, Bi/TriLinProlongationP1, SetBC2D/3D with UserBC2D/3D,
Interpolate2D) and their composition (MultigridIterations, AFASVcycle,
LevelRelax, FillDown, ErrorAFAS and the per-patch functions of
afasroutines.f90; SetGhost, InterpolateCoarseFine, TransferBC, GhostOverlap,
SetBC and GetCoarseGhostPoints of boundary.f90).  This module parses those
routines from the reference files and executes them with numpy in IEEE double
precision (the reference builds with -fdefault-real-8), evaluating every
expression left to right as written, every array statement's right-hand side
before its assignment, and SUM sequentially in array element order.

The tree module (TreeOps) is pointer code and is not interpreted: a caller
supplies `tree`, an object whose on(level) lists the level's nodeinfo records
in ApplyOnLevel order, and the interpreter provides ApplyOnLevel,
ApplyOnLevelPairs (each grid with every later one) and GetParentInfo
(lib/treeops.f90:536-610) over it.  Records are Python objects whose
attributes are the nodeinfo components.  A caller may also stand in for a
called routine (`stubs`: MakeNewGrid, to record the boxes NewSubGrids makes).
Also covered: DO WHILE, a DO without loop control (left by EXIT), WHERE
without ELSEWHERE, ALLOCATE / DEALLOCATE of integer arrays, and the pointer
statements of a linked list of derived-type scalars: ALLOCATE of a pointer
(a new record from the caller's factory for that variable, `derived`),
pointer assignment `p => q`, NULLIFY and ASSOCIATED.  Not supported (and not
needed): character data, implicit typing.

Only make_golden.py imports this module, in a container that has the
reference source; the tests read the fixtures it wrote.
"""
from __future__ import annotations

import re

import numpy as np

# ---- lexer ----------------------------------------------------------------------

_TOKEN = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([eEdD][+-]?\d+)?)
  | (?P<dotop>\.(and|or|not|true|false|eq|ne|lt|le|gt|ge)\.)
  | (?P<name>[A-Za-z_][A-Za-z_0-9]*)
  | (?P<op>\*\*|==|/=|<=|>=|::|[-+*/(),:=<>%])
  | (?P<ws>\s+)
""", re.X | re.I)


def tokenize(s: str) -> list:
    out, pos = [], 0
    while pos < len(s):
        m = _TOKEN.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot lex: {s[pos:pos + 30]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        text = m.group(kind)
        if kind == "num":
            t = text.lower().replace("d", "e")
            val = float(t) if ("." in t or "e" in t) else int(t)
            out.append(("num", val))
        elif kind == "dotop":
            out.append(("op", text.lower()))
        elif kind == "name":
            out.append(("name", text.lower()))
        else:
            out.append(("op", text))
    return out


def logical_lines(src: str) -> list:
    """Source lines with comments removed, continuations joined and ';'
    statement separators split."""
    lines, cur = [], ""
    for raw in src.splitlines():
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        stripped = line.strip()
        if stripped.startswith("&"):
            stripped = stripped[1:]
        if stripped.endswith("&"):
            cur += stripped[:-1] + " "
            continue
        cur += stripped
        for part in cur.split(";"):
            if part.strip():
                lines.append(part.strip())
        cur = ""
    return lines


# ---- arrays with Fortran bounds -----------------------------------------------

class FArray:
    """A numpy array (column-major semantics, any lower bounds)."""

    def __init__(self, data: np.ndarray, lb):
        self.data = data
        self.lb = tuple(lb)

    @property
    def shape(self):
        return self.data.shape


def rebase(a, lb):
    if isinstance(a, FArray):
        return FArray(a.data, lb)
    return FArray(np.asarray(a), lb)


# ---- expressions ---------------------------------------------------------------

class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else ("eof", None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise SyntaxError(f"expected {val!r}, got {tok!r}")
        self.i += 1
        return tok

    # precedence: .or. < .and. < .not. < relational < +- < */ < unary < **
    def expr(self):
        node = self.and_()
        while self.peek()[1] == ".or.":
            self.take()
            node = ("bin", ".or.", node, self.and_())
        return node

    def and_(self):
        node = self.not_()
        while self.peek()[1] == ".and.":
            self.take()
            node = ("bin", ".and.", node, self.not_())
        return node

    def not_(self):
        if self.peek()[1] == ".not.":
            self.take()
            return ("not", self.not_())
        return self.rel()

    def rel(self):
        node = self.add()
        ops = {"==": "==", "/=": "/=", "<": "<", ">": ">", "<=": "<=", ">=": ">=",
               ".eq.": "==", ".ne.": "/=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}
        if self.peek()[1] in ops:
            op = ops[self.take()[1]]
            node = ("bin", op, node, self.add())
        return node

    def add(self):
        if self.peek()[1] in ("+", "-"):  # leading sign: applies to the first term
            op = self.take()[1]
            node = self.mul()
            if op == "-":
                node = ("neg", node)
        else:
            node = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            node = ("bin", op, node, self.mul())
        return node

    def mul(self):
        node = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            node = ("bin", op, node, self.power())
        return node

    def power(self):
        base = self.primary()
        if self.peek()[1] == "**":
            self.take()
            return ("bin", "**", base, self.power())
        return base

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return ("num", val)
        if val in (".true.", ".false."):
            self.take()
            return ("num", val == ".true.")
        if val == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return e
        if kind == "name":
            self.take()
            while self.peek()[1] == "%":  # component chain a%b%c -> one name
                self.take()
                val = val + "%" + self.take()[1]
            if self.peek()[1] == "(":
                self.take()
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.subscript())
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return ("ref", val, args)
            return ("var", val)
        raise SyntaxError(f"unexpected token {self.peek()!r}")

    def subscript(self):
        """An argument or a section triplet lo:hi[:stride] (parts optional)."""
        lo = hi = st = None
        if self.peek()[1] != ":":
            lo = self.expr()
            if self.peek()[1] != ":":
                return lo
        self.take(":")
        if self.peek()[1] not in (",", ")", ":"):
            hi = self.expr()
        if self.peek()[1] == ":":
            self.take()
            st = self.expr()
        return ("sec", lo, hi, st)


def parse_expr(s: str):
    p = Parser(tokenize(s))
    e = p.expr()
    if p.peek()[0] != "eof":
        raise SyntaxError(f"trailing tokens in {s!r}")
    return e


# ---- routines ---------------------------------------------------------------------

class Routine:
    def __init__(self, name, kind, args, result, decls, body, elemental):
        self.name, self.kind, self.args, self.result = name, kind, args, result
        self.decls, self.body, self.elemental = decls, body, elemental


_HEAD = re.compile(r"^(?:(elemental|recursive|pure)\s+)?(?:(integer|real|logical)\s+)?"
                   r"(subroutine|function)\s+(\w+)\s*(?:\(([^)]*)\))?\s*"
                   r"(?:result\s*\(\s*(\w+)\s*\))?\s*$", re.I)


def extract_routines(src: str) -> dict:
    lines = logical_lines(src)
    out, i = {}, 0
    while i < len(lines):
        m = _HEAD.match(lines[i])
        if not m:
            i += 1
            continue
        elemental = (m.group(1) or "").lower() == "elemental"
        kind = m.group(3).lower()
        name = m.group(4).lower()
        args = [a.strip().lower() for a in (m.group(5) or "").split(",") if a.strip()]
        result = (m.group(6) or (name if kind == "function" else "")).lower()
        j = i + 1
        while not re.match(rf"^end\s+{kind}\b", lines[j], re.I):
            j += 1
        decls, body = [], []
        for ln in lines[i + 1:j]:
            low = ln.lower()
            if re.match(r"^(use|implicit)\b", low):
                continue
            if re.match(r"^(real|integer|logical|double\s+precision|type\s*\()", low) and "::" in ln:
                decls.append(ln)
            elif re.match(r"^(real|integer|logical)\s+\w", low) and "=" not in ln.split("::")[0]:
                decls.append(ln)
            else:
                body.append(ln)
        out[name] = Routine(name, kind, args, result, decls, body, elemental)
        i = j + 1
    return out


def parse_module_parameters(src: str) -> dict:
    """`real, parameter :: name = expr` constants of a module."""
    consts = {}
    for ln in logical_lines(src):
        m = re.match(r"^real\s*,\s*parameter\s*::\s*(\w+)\s*=\s*(.+)$", ln, re.I)
        if m:
            consts[m.group(1).lower()] = m.group(2)
    return consts


class Record:
    """A derived-type value (nodeinfo, funcparam): components are attributes."""

    def __init__(self, **comps):
        self.__dict__.update(comps)


_MISSING = object()


class Interp:
    def __init__(self, routines: dict, globals_: dict, tree=None):
        self.routines = routines
        self.globals = dict(globals_)
        self.tree = tree        # TreeOps stand-in: tree.on(level) -> records
        self.current = []       # ApplyOnLevel's current record (GetParentInfo)
        self.printed = []       # numeric items of every executed PRINT
        self.stubs = {}         # name -> Python callable standing in for a CALL
        self.derived = {}       # pointer variable -> factory of a new target record

    def lookup(self, name, env):
        """A variable, or a component chain a%b%c, from the locals, then the
        module variables; _MISSING when the base name is neither."""
        base, *comps = name.split("%")
        if base in env:
            obj = env[base]
        elif base in self.globals:
            obj = self.globals[base]
        else:
            return _MISSING
        for c in comps:
            obj = getattr(obj, c)
        return obj

    # -- evaluation -------------------------------------------------------------
    def ev(self, node, env):
        k = node[0]
        if k == "num":
            return node[1]
        if k == "var":
            name = node[1]
            v = self.lookup(name, env)
            if v is _MISSING:
                raise NameError(name)
            return v.data if isinstance(v, FArray) else v
        if k == "neg":
            return -self.ev(node[1], env)
        if k == "not":
            return np.logical_not(self.ev(node[1], env))
        if k == "bin":
            op = node[1]
            a = self.ev(node[2], env)
            b = self.ev(node[3], env)
            if op == "+":
                return a + b
            if op == "-":
                return a - b
            if op == "*":
                return a * b
            if op == "/":
                if np.asarray(a).dtype.kind in "iu" and np.asarray(b).dtype.kind in "iu":
                    q = np.abs(a) // np.abs(b)  # integer division truncates
                    return np.where((np.asarray(a) >= 0) == (np.asarray(b) >= 0), q, -q) \
                        if np.ndim(q) else (q if (a >= 0) == (b >= 0) else -q)
                return a / b
            if op == "**":
                if isinstance(b, (int, np.integer)) and b >= 0:
                    r = a
                    for _ in range(b - 1):
                        r = r * a
                    return r if b > 0 else 1.0
                return a ** b
            if op == "==":
                return a == b
            if op == "/=":
                return a != b
            if op == "<":
                return a < b
            if op == ">":
                return a > b
            if op == "<=":
                return a <= b
            if op == ">=":
                return a >= b
            if op == ".and.":
                return np.logical_and(a, b)
            if op == ".or.":
                return np.logical_or(a, b)
        if k == "ref":
            return self.ref(node, env)
        raise ValueError(node)

    def index_tuple(self, arr: FArray, subs, env):
        idx = []
        for d, s in enumerate(subs):
            lb = arr.lb[d]
            n = arr.data.shape[d]
            if isinstance(s, tuple) and s[0] == "sec":
                lo = lb if s[1] is None else self.ev(s[1], env)
                hi = lb + n - 1 if s[2] is None else self.ev(s[2], env)
                st = 1 if s[3] is None else self.ev(s[3], env)
                if st > 0:
                    stop = hi - lb + 1
                    idx.append(slice(lo - lb, max(stop, lo - lb), st))
                else:
                    raise NotImplementedError("negative strides")
            else:
                i = int(self.ev(s, env))
                if not (lb <= i < lb + n):
                    raise IndexError(f"index {i} outside {lb}:{lb + n - 1}")
                idx.append(i - lb)
        return tuple(idx)

    def ref(self, node, env):
        _, name, subs = node
        arr = self.lookup(name, env)
        if isinstance(arr, FArray):
            return arr.data[self.index_tuple(arr, subs, env)]
        return self.call_function(name, subs, env)

    def section_actual(self, s, env):
        """An actual argument: arrays and sections keep their storage (views)."""
        if s[0] == "var":
            v = self.lookup(s[1], env)
            if isinstance(v, FArray):
                return FArray(v.data, (1,) * v.data.ndim)
            return v
        if s[0] == "ref":
            arr = self.lookup(s[1], env)
            if isinstance(arr, FArray):
                view = arr.data[self.index_tuple(arr, s[2], env)]
                if isinstance(view, np.ndarray) and view.ndim > 0:
                    return FArray(view, (1,) * view.ndim)
                return view
        v = self.ev(s, env)
        if isinstance(v, np.ndarray) and v.ndim > 0:
            return FArray(v, (1,) * v.ndim)
        return v

    def call_function(self, name, subs, env):
        if name == "associated":
            return self.lookup(subs[0][1], env) is not None
        if name == "size":
            a = self.section_actual(subs[0], env)
            d = int(self.ev(subs[1], env)) if len(subs) > 1 else None
            return a.data.shape[d - 1] if d else a.data.size
        if name == "modulo":
            a, p = self.ev(subs[0], env), self.ev(subs[1], env)
            return a % p
        if name == "mod":
            a, p = self.ev(subs[0], env), self.ev(subs[1], env)
            return int(np.fmod(a, p))
        if name in ("max", "min"):
            vals = [self.ev(s, env) for s in subs]
            f = np.maximum if name == "max" else np.minimum
            r = vals[0]
            for v in vals[1:]:
                r = f(r, v)
            return r
        if name == "abs":
            return np.abs(self.ev(subs[0], env))
        if name == "sqrt":
            return np.sqrt(self.ev(subs[0], env))
        if name == "sum":  # sequential, in array element order
            a = np.asarray(self.ev(subs[0], env))
            acc = np.float64(0.0) if a.dtype.kind == "f" else 0
            for x in np.ravel(a, order="F"):
                acc = acc + x
            return acc
        if name == "product":
            a = np.asarray(self.ev(subs[0], env))
            acc = 1
            for x in np.ravel(a, order="F"):
                acc = acc * x
            return acc
        if name == "maxval":
            return np.max(self.ev(subs[0], env))
        if name == "minval":
            return np.min(self.ev(subs[0], env))
        if name == "any":
            return bool(np.any(self.ev(subs[0], env)))
        if name == "getparentinfo":  # GetParentInfo(parent) -> err_ok
            env[subs[0][1]] = self.current[-1].parent
            return 0
        if name in ("real", "dble"):
            return np.float64(self.ev(subs[0], env)) if np.isscalar(self.ev(subs[0], env)) else \
                self.ev(subs[0], env).astype(np.float64)
        r = self.routines[name]
        actuals = [self.section_actual(s, env) for s in subs]
        if r.elemental:
            return self.run_elemental(r, actuals)
        return self.run(r, actuals)

    def run_elemental(self, r, actuals):
        vals = [a.data if isinstance(a, FArray) else a for a in actuals]
        env = {an: np.asarray(v, dtype=np.float64) if not np.isscalar(v) else v
               for an, v in zip(r.args, vals)}
        # Scalar temporaries of the body broadcast over the argument's shape.
        self.exec_block(r.body, env)
        res = env[r.result]
        shape = np.broadcast(*[np.asarray(v) for v in vals]).shape
        return np.broadcast_to(np.asarray(res, dtype=np.float64), shape).copy() if shape else res

    # -- declarations ---------------------------------------------------------------
    def declare(self, r, env):
        for d in r.decls:
            head, names = d.split("::", 1)
            attrs = [a.strip() for a in split_top(head, ",")]
            base = attrs[0].lower()
            dims = None
            for a in attrs[1:]:
                m = re.match(r"dimension\s*\((.*)\)\s*$", a, re.I)
                if m:
                    dims = m.group(1)
            for item in split_top(names, ","):
                item = item.strip()
                m = re.match(r"(\w+)\s*(\((.*)\))?\s*(=\s*(.+))?$", item)
                nm = m.group(1).lower()
                local_dims = m.group(3) or dims
                init = m.group(5)
                if base.startswith("type"):
                    if nm not in r.args:  # funcparam locals; nodeinfo pointers unset
                        env[nm] = Record(iswitch=0) if "funcparam" in base else None
                    continue
                if nm in r.args:
                    a = env.get(nm)
                    if local_dims is not None and isinstance(a, FArray):
                        lbs = []
                        for k, spec in enumerate(split_top(local_dims, ",")):
                            spec = spec.strip()
                            if ":" in spec:
                                lo = spec.split(":")[0].strip()
                                lbs.append(int(self.ev(parse_expr(lo), env)) if lo else 1)
                            else:
                                lbs.append(1)
                        env[nm] = FArray(a.data, lbs)
                    continue
                if local_dims is not None and any(a.lower() == "allocatable" for a in attrs):
                    env[nm] = None  # created by ALLOCATE
                    continue
                if local_dims is not None:
                    lbs, shape = [], []
                    for spec in split_top(local_dims, ","):
                        spec = spec.strip()
                        if ":" in spec:
                            lo_s, hi_s = spec.split(":", 1)
                            lo = int(self.ev(parse_expr(lo_s), env))
                            hi = int(self.ev(parse_expr(hi_s), env))
                        else:
                            lo, hi = 1, int(self.ev(parse_expr(spec), env))
                        lbs.append(lo)
                        shape.append(max(hi - lo + 1, 0))
                    dt = np.float64 if base.startswith("real") else (
                        np.int64 if base.startswith("integer") else bool)
                    env[nm] = FArray(np.full(shape, np.nan if dt == np.float64 else 0, dtype=dt,
                                             order="F"), lbs)
                elif init is not None:
                    env[nm] = self.ev(parse_expr(init), env)
                else:
                    env[nm] = 0.0 if base.startswith("real") else 0

    def run(self, r, actuals):
        env = {}
        for an, av in zip(r.args, actuals):
            env[an] = av
        self.declare(r, env)
        try:
            self.exec_block(r.body, env)
        except _Return:
            pass
        if r.kind == "function":
            v = env[r.result]
            return v.data if isinstance(v, FArray) else v
        return None

    # -- statements -----------------------------------------------------------------
    def exec_block(self, lines, env):
        i = 0
        while i < len(lines):
            i = self.exec_stmt(lines, i, env)

    def find_end(self, lines, i, opener, closer, middles=()):
        """Index of the matching closer (and of the middle keywords) for the
        construct opened at lines[i]."""
        depth, mids = 0, []
        for j in range(i, len(lines)):
            low = lines[j].lower()
            if opener(low):
                depth += 1
            elif closer(low):
                depth -= 1
                if depth == 0:
                    return j, mids
            elif depth == 1 and any(mm(low) for mm in middles):
                mids.append(j)
        raise SyntaxError(f"unterminated construct at {lines[i]!r}")

    def exec_stmt(self, lines, i, env):
        ln = lines[i]
        low = ln.lower()
        lab = re.match(r"^(\w+)\s*:\s*(do\b.*)$", ln, re.I)
        if lab:
            ln = lab.group(2)
            low = ln.lower()
        if re.match(r"^do\s+while\s*\(", low):
            is_do = lambda s: bool(re.match(r"^(\w+\s*:\s*)?do\b", s))
            is_end = lambda s: bool(re.match(r"^end\s*do\b", s))
            end, _ = self.find_end(lines, i, is_do, is_end)
            cond_s, _ = split_paren(ln[ln.lower().index("while") + 5:].strip())
            body = lines[i + 1:end]
            name = lab.group(1).lower() if lab else None
            while bool(self.ev(parse_expr(cond_s), env)):
                try:
                    self.exec_block(body, env)
                except _Cycle as c:
                    if c.name not in (None, name):
                        raise
                except _Exit as e:
                    if e.name not in (None, name):
                        raise
                    break
            return end + 1
        if re.match(r"^where\s*\(", low):
            # WHERE (mask) ... END WHERE (no ELSEWHERE): each assignment of
            # the block applied where the mask holds.
            is_w = lambda s: bool(re.match(r"^where\s*\(", s)) and not \
                split_paren(s[5:].strip())[1].strip()
            is_end = lambda s: bool(re.match(r"^end\s*where\b", s))
            end, _ = self.find_end(lines, i, is_w, is_end)
            mask_s, _ = split_paren(ln[5:].strip())
            mask = np.asarray(self.ev(parse_expr(mask_s), env), dtype=bool)
            for st in lines[i + 1:end]:
                lhs_s, rhs_s = split_assign(st)
                rhs = np.broadcast_to(np.asarray(self.ev(parse_expr(rhs_s), env)), mask.shape)
                lhs = parse_expr(lhs_s)
                arr = self.lookup(lhs[1], env)
                view = arr.data[self.index_tuple(arr, lhs[2], env)] if lhs[0] == "ref" else arr.data
                view[mask] = rhs[mask]
            return end + 1
        if re.match(r"^allocate\s*\(", low):
            inner, _ = split_paren(ln[8:].strip())
            for item in split_top(inner, ","):
                item = item.strip()
                if re.match(r"^stat\s*=", item, re.I):
                    env[item.split("=", 1)[1].strip().lower()] = 0
                    continue
                m = re.match(r"^(\w+)\s*\((.*)\)$", item)
                if m is None:  # a pointer to a derived-type scalar
                    self.assign_ref(item.lower(), self.derived[item.lower()](), env)
                    continue
                nm, dims = m.group(1).lower(), m.group(2)
                lbs, shape = [], []
                for spec in split_top(dims, ","):
                    lo_s, hi_s = spec.split(":", 1) if ":" in spec else ("1", spec)
                    lo = int(self.ev(parse_expr(lo_s), env))
                    hi = int(self.ev(parse_expr(hi_s), env))
                    lbs.append(lo)
                    shape.append(max(hi - lo + 1, 0))
                env[nm] = FArray(np.zeros(shape, dtype=np.int64, order="F"), lbs)
            return i + 1
        if re.match(r"^deallocate\s*\(", low):
            inner, _ = split_paren(ln[10:].strip())
            for item in split_top(inner, ","):
                item = item.strip()
                if re.match(r"^stat\s*=", item, re.I):
                    env[item.split("=", 1)[1].strip().lower()] = 0
            return i + 1
        if re.match(r"^do\s*$", low):
            # DO without loop control, left by EXIT.
            is_do = lambda s: bool(re.match(r"^(\w+\s*:\s*)?do\b", s))
            is_end = lambda s: bool(re.match(r"^end\s*do\b", s))
            end, _ = self.find_end(lines, i, is_do, is_end)
            body = lines[i + 1:end]
            name = lab.group(1).lower() if lab else None
            while True:
                try:
                    self.exec_block(body, env)
                except _Cycle as c:
                    if c.name not in (None, name):
                        raise
                except _Exit as e:
                    if e.name not in (None, name):
                        raise
                    return end + 1
        if re.match(r"^nullify\s*\(", low):
            inner, _ = split_paren(ln[7:].strip())
            for item in split_top(inner, ","):
                self.assign_ref(item.strip().lower(), None, env)
            return i + 1
        if "=>" in ln:
            # Pointer assignment: the left side names the record the right
            # side names (or none, for null()).
            lhs_s, rhs_s = (x.strip().lower() for x in ln.split("=>", 1))
            target = None if rhs_s.replace(" ", "") == "null()" else self.lookup(rhs_s, env)
            if target is _MISSING:
                raise NameError(rhs_s)
            self.assign_ref(lhs_s, target, env)
            return i + 1
        if re.match(r"^do\b", low):
            is_do = lambda s: bool(re.match(r"^(\w+\s*:\s*)?do\b", s))
            is_end = lambda s: bool(re.match(r"^end\s*do\b", s))
            end, _ = self.find_end(lines, i, is_do, is_end)
            m = re.match(r"^do\s+(\w+)\s*=\s*(.+)$", ln, re.I)
            var = m.group(1).lower()
            parts = split_top(m.group(2), ",")
            lo = int(self.ev(parse_expr(parts[0]), env))
            hi = int(self.ev(parse_expr(parts[1]), env))
            st = int(self.ev(parse_expr(parts[2]), env)) if len(parts) > 2 else 1
            body = lines[i + 1:end]
            name = lab.group(1).lower() if lab else None
            v = lo
            while (st > 0 and v <= hi) or (st < 0 and v >= hi):
                env[var] = v
                try:
                    self.exec_block(body, env)
                except _Cycle as c:
                    if c.name not in (None, name):
                        raise
                except _Exit as e:
                    if e.name not in (None, name):
                        raise
                    return end + 1  # the DO variable keeps its value
                v += st
            env[var] = v
            return end + 1
        if re.match(r"^if\s*\(", low):
            cond_s, rest = split_paren(ln[2:].strip())
            if rest.strip().lower() == "then":
                is_if = lambda s: bool(re.match(r"^if\s*\(.*\)\s*then$", s))
                is_end = lambda s: bool(re.match(r"^end\s*if\b", s))
                is_mid = lambda s: bool(re.match(r"^else\b", s))
                end, mids = self.find_end(lines, i, is_if, is_end, (is_mid,))
                branches, start, cond = [], i + 1, cond_s
                for mj in mids + [end]:
                    branches.append((cond, lines[start:mj]))
                    if mj == end:
                        break
                    m2 = re.match(r"^else\s*if\s*\((.*)\)\s*then$", lines[mj], re.I)
                    cond = m2.group(1) if m2 else None
                    start = mj + 1
                for cond, blk in branches:
                    if cond is None or bool(self.ev(parse_expr(cond), env)):
                        self.exec_block(blk, env)
                        break
                return end + 1
            if bool(self.ev(parse_expr(cond_s), env)):
                self.exec_stmt([rest.strip()], 0, env)
            return i + 1
        if re.match(r"^select\s+case\b", low):
            is_sel = lambda s: bool(re.match(r"^select\s+case\b", s))
            is_end = lambda s: bool(re.match(r"^end\s*select\b", s))
            is_case = lambda s: bool(re.match(r"^case\b", s))
            end, mids = self.find_end(lines, i, is_sel, is_end, (is_case,))
            sel = self.ev(parse_expr(ln[ln.index("(") + 1:ln.rindex(")")]), env)
            for a, mj in enumerate(mids):
                stop = mids[a + 1] if a + 1 < len(mids) else end
                spec = lines[mj][4:].strip()
                if spec.lower() == "default" or self.case_match(spec, sel, env):
                    self.exec_block(lines[mj + 1:stop], env)
                    break
            return end + 1
        if re.match(r"^cycle\b", low):
            parts = low.split()
            raise _Cycle(parts[1] if len(parts) > 1 else None)
        if re.match(r"^exit\b", low):
            parts = low.split()
            raise _Exit(parts[1] if len(parts) > 1 else None)
        if re.match(r"^print\s*\*\s*,", low):
            items = split_print(ln[ln.index(",") + 1:])
            self.printed.append(tuple(self.ev(parse_expr(it), env) for it in items
                                      if not it.strip().startswith(("'", '"'))))
            return i + 1
        if re.match(r"^\d+\s+format\b", low):  # FORMAT statements do nothing
            return i + 1
        if low in ("continue", "return") or re.match(r"^(print|write)\b", low):
            if low == "return":
                raise _Return()
            return i + 1
        if re.match(r"^stop\b", low):
            raise RuntimeError("reference executed STOP")
        if re.match(r"^call\b", low):
            node = parse_expr(ln[4:].strip())
            if node[1] in self.stubs:  # a routine the caller stands in for
                self.stubs[node[1]](*[self.section_actual(x, env) for x in node[2]])
                return i + 1
            if node[1] in ("applyonlevel", "applyonlevelpairs"):
                level = int(self.ev(node[2][0], env))
                fn = self.routines[node[2][1][1]]
                param = self.lookup(node[2][2][1], env)
                self.apply_on_level(level, fn, param, pairs=node[1] == "applyonlevelpairs")
                return i + 1
            r = self.routines[node[1]]
            self.run(r, [self.section_actual(s, env) for s in node[2]])
            return i + 1
        # Assignment.
        lhs_s, rhs_s = split_assign(ln)
        rhs = self.ev(parse_expr(rhs_s), env)
        if isinstance(rhs, np.ndarray):
            rhs = rhs.copy()
        lhs = parse_expr(lhs_s)
        if lhs[0] == "var":
            name = lhs[1]
            if "%" in name:
                owner_s, comp = name.rsplit("%", 1)
                owner, scope, key = self.lookup(owner_s, env), None, comp
            elif name in env or name not in self.globals:
                owner, scope, key = None, env, name
            else:  # a module variable
                owner, scope, key = None, self.globals, name
            cur = getattr(owner, key) if owner is not None else scope.get(key)
            if isinstance(cur, FArray):
                cur.data[...] = rhs
            elif owner is not None:
                setattr(owner, key, rhs)
            else:
                scope[key] = rhs
        else:
            arr = self.lookup(lhs[1], env)
            arr.data[self.index_tuple(arr, lhs[2], env)] = rhs
        return i + 1

    def assign_ref(self, name, target, env):
        """Makes variable or component `name` refer to `target`."""
        if "%" in name:
            owner_s, comp = name.rsplit("%", 1)
            setattr(self.lookup(owner_s, env), comp, target)
        elif name in env or name not in self.globals:
            env[name] = target
        else:
            self.globals[name] = target

    def apply_on_level(self, level, fn, param, pairs):
        """ApplyOnLevel / ApplyOnLevelPairs (lib/treeops.f90:536-610): fn on
        every record of the level in list order (pairs: each record with every
        later one); a nonzero return ends the traversal."""
        recs = self.tree.on(level)
        for a, rec in enumerate(recs):
            for other in (recs[a + 1:] if pairs else [None]):
                self.current.append(rec)
                try:
                    args = [rec, other, param] if pairs else [rec, param]
                    code = self.run(fn, args)
                finally:
                    self.current.pop()
                if code:
                    self.tree.errcode = code
                    return

    def case_match(self, spec, sel, env):
        inner = spec[spec.index("(") + 1:spec.rindex(")")]
        for item in split_top(inner, ","):
            if ":" in item:
                lo, hi = item.split(":")
                if int(self.ev(parse_expr(lo), env)) <= sel <= int(self.ev(parse_expr(hi), env)):
                    return True
            elif sel == self.ev(parse_expr(item), env):
                return True
        return False


class _Cycle(Exception):
    def __init__(self, name):
        self.name = name


class _Return(Exception):
    pass


class _Exit(Exception):
    def __init__(self, name):
        self.name = name


def split_print(s: str) -> list:
    """The output items of a list-directed PRINT (commas outside quotes and
    parentheses)."""
    out, depth, cur, quote = [], 0, "", None
    for ch in s:
        if quote:
            quote = None if ch == quote else quote
        elif ch in "'\"":
            quote = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "," and depth == 0:
            out.append(cur)
            cur = ""
            continue
        cur += ch
    out.append(cur)
    return [o for o in out if o.strip()]


def split_top(s: str, sep: str) -> list:
    """Split at `sep` outside parentheses."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    out.append(cur)
    return out


def split_paren(s: str):
    """'(cond) rest' -> ('cond', 'rest')."""
    depth = 0
    for k, ch in enumerate(s):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return s[1:k], s[k + 1:]
    raise SyntaxError(s)


def split_assign(s: str):
    depth = 0
    for k, ch in enumerate(s):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0 and s[k - 1] not in "<>/=" and s[k + 1] != "=":
            return s[:k], s[k + 1:]
    raise SyntaxError(f"not an assignment: {s!r}")

"""Parser of the Fortran 90 subset run by the oracle's source runner.

TEST INFRASTRUCTURE ONLY (see oracle/f90/__init__.py). Modules are read in
full at the specification level (use statements, access statements,
declarations, derived types, generic interfaces, procedure headers); the
executable statements of a procedure are parsed only when the procedure is
needed, so constructs outside the subset in unused procedures do no harm. A
construct outside the subset in a needed procedure raises FortranSubsetError
naming file and line.

Expression nodes (tuples):
  ('int', value)  ('real', value, kind)  ('str', text)  ('log', bool)
  ('name', n)  ('ref', base, [args])  ('comp', base, name)
  ('un', op, e)  ('bin', op, a, b)  ('sec', lo, hi, step)  ('kw', name, e)
  ('cons', [elements])
Statement nodes: see Parser.statement.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .lex import FortranSubsetError, logical_lines, tokenize


# --------------------------------------------------------------------------- tokens
class Toks:
    def __init__(self, toks, where):
        self.t = toks
        self.i = 0
        self.where = where
        self.bind_c = None

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else ("eof", None)

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def at(self, kind, val=None, k=0):
        tk = self.peek(k)
        return tk[0] == kind and (val is None or tk[1] == val)

    def accept(self, kind, val=None):
        if self.at(kind, val):
            return self.next()
        return None

    def expect(self, kind, val=None):
        if not self.at(kind, val):
            self.fail(f"expected {val or kind}, found {self.peek()[1]!r}")
        return self.next()

    def done(self):
        return self.i >= len(self.t)

    def fail(self, msg):
        raise FortranSubsetError(f"{self.where}: {msg}")


# --------------------------------------------------------------------------- literals
# integer named constants of the modules being read (kind parameters such as KREAL); the reader
# and the body parser point this at the program's table before they parse
_KINDS: dict = {}


def real_literal(text: str):
    """(value, kind) of a real literal: 'd' exponents and _kreal/_8 suffixes are double; a
    literal without either is default (single) precision, rounded to binary32 as a compiler
    stores it, then widened exactly wherever it meets a double."""
    body, _, suffix = text.partition("_")
    low = body.lower()
    if "d" in low:
        return float(low.replace("d", "e")), 8
    if suffix:
        if suffix.lower() in ("kreal", "8", "dp", "rk"):
            return float(low), 8
        if suffix.lower() == "4":
            return float(np.float32(float(low))), 4
        k = _KINDS.get(suffix.lower())
        if k == 8:
            return float(low), 8
        if k == 4:
            return float(np.float32(float(low))), 4
        raise FortranSubsetError(f"unknown real kind suffix in {text}")
    return float(np.float32(float(low))), 4


def int_literal(text: str) -> int:
    return int(text.partition("_")[0])


# --------------------------------------------------------------------------- expressions
_REL = {"==": "==", "/=": "/=", "<": "<", "<=": "<=", ">": ">", ">=": ">=",
        "eq": "==", "ne": "/=", "lt": "<", "le": "<=", "gt": ">", "ge": ">="}


def parse_expr(ts: Toks):
    return _equiv(ts)


def _equiv(ts):
    e = _or(ts)
    while ts.at("dot", "eqv") or ts.at("dot", "neqv"):
        op = ts.next()[1]
        e = ("bin", op, e, _or(ts))
    return e


def _or(ts):
    e = _and(ts)
    while ts.accept("dot", "or"):
        e = ("bin", "or", e, _and(ts))
    return e


def _and(ts):
    e = _not(ts)
    while ts.accept("dot", "and"):
        e = ("bin", "and", e, _not(ts))
    return e


def _not(ts):
    if ts.accept("dot", "not"):
        return ("un", "not", _not(ts))
    return _rel(ts)


def _rel(ts):
    e = _concat(ts)
    tk = ts.peek()
    if (tk[0] == "op" and tk[1] in _REL) or (tk[0] == "dot" and tk[1] in _REL):
        ts.next()
        e = ("bin", _REL[tk[1]], e, _concat(ts))
    return e


def _concat(ts):
    e = _add(ts)
    while ts.accept("op", "//"):
        e = ("bin", "//", e, _add(ts))
    return e


def _add(ts):
    # level-2 expression: [sign] add-operand { add-op add-operand }; the sign applies to the
    # first add-operand as a whole (-a*b is -(a*b), -a**2 is -(a**2))
    if ts.at("op", "-") or ts.at("op", "+"):
        op = ts.next()[1]
        e = _mul(ts)
        if op == "-":
            e = ("un", "-", e)
    else:
        e = _mul(ts)
    while ts.at("op", "+") or ts.at("op", "-"):
        op = ts.next()[1]
        e = ("bin", op, e, _mul(ts))
    return e


def _mul(ts):
    e = _pow(ts)
    while ts.at("op", "*") or ts.at("op", "/"):
        op = ts.next()[1]
        e = ("bin", op, e, _pow(ts))
    return e


def _pow(ts):
    base = _unary_in_operand(ts)
    if ts.accept("op", "**"):
        return ("bin", "**", base, _pow(ts))  # right associative
    return base


def _unary_in_operand(ts):
    # extension accepted by common compilers: a sign directly after a binary operator (a*-b)
    if ts.at("op", "-") or ts.at("op", "+"):
        op = ts.next()[1]
        e = _pow(ts)
        return ("un", "-", e) if op == "-" else e
    return _primary(ts)


def _primary(ts):
    tk = ts.next()
    kind, val = tk
    if kind == "int":
        return ("int", int_literal(val))
    if kind == "real":
        v, k = real_literal(val)
        return ("real", v, k)
    if kind == "str":
        return ("str", val)
    if kind == "dot" and val in ("true", "false"):
        return ("log", val == "true")
    if kind == "op" and val == "(":
        e = parse_expr(ts)
        ts.expect("op", ")")
        return ("paren", e)
    if kind == "op" and val in ("(/", "["):
        close = "/)" if val == "(/" else "]"
        elems = []
        if not ts.at("op", close):
            elems.append(parse_expr(ts))
            while ts.accept("op", ","):
                elems.append(parse_expr(ts))
        ts.expect("op", close)
        return ("cons", elems)
    if kind == "name":
        return _postfix(ts, ("name", val))
    ts.fail(f"unexpected token {val!r} in expression")


def _postfix(ts, e):
    while True:
        if ts.accept("op", "("):
            args = []
            if not ts.at("op", ")"):
                args.append(_arg(ts))
                while ts.accept("op", ","):
                    args.append(_arg(ts))
            ts.expect("op", ")")
            e = ("ref", e, args)
        elif ts.accept("op", "%"):
            e = ("comp", e, ts.expect("name")[1])
        else:
            return e


def _arg(ts):
    # keyword argument, section triplet, or expression
    if ts.at("name") and ts.at("op", "=", 1):
        name = ts.next()[1]
        ts.next()
        return ("kw", name, parse_expr(ts))
    if ts.at("op", ":") or ts.at("op", "::"):
        lo = None
    else:
        lo = parse_expr(ts)
        if not (ts.at("op", ":") or ts.at("op", "::")):
            return lo
    if ts.accept("op", "::"):  # a::s (empty upper bound)
        return ("sec", lo, None, parse_expr(ts))
    ts.expect("op", ":")
    hi = None
    if not (ts.at("op", ",") or ts.at("op", ")") or ts.at("op", ":")):
        hi = parse_expr(ts)
    step = None
    if ts.accept("op", ":"):
        step = parse_expr(ts)
    return ("sec", lo, hi, step)


# --------------------------------------------------------------------------- declarations
@dataclass
class VType:
    base: str              # 'real' 'integer' 'logical' 'character' 'type'
    kind: int = 0          # real: 8 or 4; integer/logical: 4
    tname: str = ""        # derived type name


@dataclass
class Var:
    name: str
    vt: VType
    shape: list | None = None   # None scalar; list of (lo, hi) expr pairs, ':' deferred, '*'
    attrs: set = field(default_factory=set)
    intent: str = ""
    init: object = None          # expression
    ptr_init: bool = False       # => null()
    where: str = ""

    @property
    def rank(self):
        return len(self.shape) if self.shape else 0


@dataclass
class TypeDef:
    name: str
    comps: dict                   # name -> Var


@dataclass
class ProcHeader:
    name: str
    kind: str                     # 'subroutine' | 'function'
    args: list
    result: str | None
    prefix_type: VType | None
    module: str
    lines: list                   # [(lineno, text)] of the body (after the header)
    path: str
    lineno: int
    parsed: object = None         # Proc once parsed


@dataclass
class Module:
    name: str
    path: str
    uses: list = field(default_factory=list)       # (module, only list | None, renames {local: remote})
    default_private: bool = False
    public: set = field(default_factory=set)
    private: set = field(default_factory=set)
    vars: dict = field(default_factory=dict)        # name -> Var
    types: dict = field(default_factory=dict)       # name -> TypeDef
    generics: dict = field(default_factory=dict)    # generic name -> [specific names]
    procs: dict = field(default_factory=dict)       # name -> ProcHeader
    includes: list = field(default_factory=list)
    cprocs: dict = field(default_factory=dict)      # name -> CProc (BIND(C) interfaces)
    namelists: dict = field(default_factory=dict)   # group -> [variable names] (programs)
    is_program: bool = False


_TYPE_KW = ("real", "integer", "logical", "character", "complex", "double")


def _is_decl(ts: Toks) -> bool:
    tk = ts.peek()
    if tk[0] != "name":
        return False
    if tk[1] in ("real", "integer", "logical", "character", "complex"):
        return True
    if tk[1] == "double" and ts.at("name", "precision", 1):
        return True
    if tk[1] == "type" and ts.at("op", "(", 1):
        return True
    return False


def _kind_value(e, consts):
    if e[0] == "int":
        return e[1]
    if e[0] == "name":
        if e[1] in consts:
            return consts[e[1]]
    if e[0] == "ref" and e[1] == ("name", "kind"):
        a = e[2][0]
        if a[0] == "real":
            return a[2]
        if a[0] == "int":
            return 4
        if a[0] == "log":
            return 4
    raise FortranSubsetError(f"cannot evaluate kind selector {e}")


def parse_typespec(ts: Toks, consts) -> VType:
    kw = ts.next()[1]
    if kw == "double":
        ts.expect("name", "precision")
        return VType("real", 8)
    if kw == "type":
        ts.expect("op", "(")
        name = ts.expect("name")[1]
        ts.expect("op", ")")
        if name == "c_ptr":  # iso_c_binding: a C address, held as an integer (None = C_NULL_PTR)
            return VType("cptr", 8)
        return VType("type", 0, name)
    if kw == "complex":
        ts.fail("complex type outside the subset")
    kind = {"real": 4, "integer": 4, "logical": 4, "character": 1}[kw]
    if ts.accept("op", "("):
        if ts.at("name") and ts.at("op", "=", 1):
            key = ts.next()[1]
            ts.next()
        else:
            key = "len" if kw == "character" else "kind"
        if ts.accept("op", "*"):
            val = None
        else:
            val = parse_expr(ts)
        ts.expect("op", ")")
        if key == "kind":
            kind = _kind_value(val, consts)
    elif kw == "character" and ts.accept("op", "*"):
        if ts.accept("op", "("):
            ts.accept("op", "*") or parse_expr(ts)
            ts.expect("op", ")")
        else:
            ts.next()
    if kw == "real" and kind not in (4, 8):
        ts.fail(f"real kind {kind} outside the subset")
    return VType(kw, kind)


def parse_arrayspec(ts: Toks) -> list:
    ts.expect("op", "(")
    dims = []
    while True:
        if ts.accept("op", ":"):
            dims.append(":")
        elif ts.accept("op", "*"):
            dims.append("*")
        else:
            lo = parse_expr(ts)
            if ts.accept("op", ":"):
                if ts.at("op", ",") or ts.at("op", ")"):
                    dims.append((lo, ":"))  # assumed shape with a lower bound
                elif ts.accept("op", "*"):
                    dims.append((lo, "*"))
                else:
                    dims.append((lo, parse_expr(ts)))
            else:
                dims.append((("int", 1), lo))
        if ts.accept("op", ")"):
            return dims
        ts.expect("op", ",")


def parse_decl(ts: Toks, consts, where) -> list[Var]:
    vt = parse_typespec(ts, consts)
    attrs, intent, dimspec = set(), "", None
    while ts.accept("op", ","):
        a = ts.expect("name")[1]
        if a == "dimension":
            dimspec = parse_arrayspec(ts)
        elif a == "intent":
            ts.expect("op", "(")
            intent = ts.expect("name")[1]
            if intent == "in" and ts.accept("name", "out"):
                intent = "inout"
            ts.expect("op", ")")
        elif a in ("pointer", "allocatable", "save", "parameter", "optional", "target", "public",
                   "private", "external", "intrinsic", "value"):
            attrs.add(a)
        else:
            ts.fail(f"attribute {a} outside the subset")
    ts.accept("op", "::")
    out = []
    while True:
        name = ts.expect("name")[1]
        shape = dimspec
        if ts.at("op", "("):
            shape = parse_arrayspec(ts)
        if ts.accept("op", "*"):  # character*len entity
            if ts.accept("op", "("):
                parse_expr(ts)
                ts.expect("op", ")")
            else:
                ts.next()
        v = Var(name, VType(vt.base, vt.kind, vt.tname), list(shape) if shape else None, set(attrs),
                intent, where=where)
        if ts.accept("op", "="):
            v.init = parse_expr(ts)
        elif ts.accept("op", "=>"):
            e = parse_expr(ts)
            if e != ("ref", ("name", "null"), []):
                ts.fail("pointer initialisation other than null()")
            v.ptr_init = True
        out.append(v)
        if not ts.accept("op", ","):
            break
    if not ts.done():
        ts.fail(f"unexpected {ts.peek()[1]!r} after declaration")
    return out


# --------------------------------------------------------------------------- module reader
_END_PROC = ("subroutine", "function")


def _header(ts: Toks, consts):
    """(kind, name, args, result, prefix type) of a procedure header, or None."""
    save = ts.i
    prefix_type = None
    while True:
        if ts.at("name", "recursive") or ts.at("name", "pure") or ts.at("name", "elemental"):
            ts.next()
        elif ts.at("name", "subroutine") or ts.at("name", "function"):
            break
        elif _is_decl(ts) and prefix_type is None:
            prefix_type = parse_typespec(ts, consts)
        else:
            ts.i = save
            return None
    kind = ts.next()[1]
    name = ts.expect("name")[1]
    args = []
    if ts.accept("op", "("):
        if not ts.at("op", ")"):
            args.append(ts.expect("name")[1])
            while ts.accept("op", ","):
                args.append(ts.expect("name")[1])
        ts.expect("op", ")")
    result = None
    if ts.accept("name", "result"):
        ts.expect("op", "(")
        result = ts.expect("name")[1]
        ts.expect("op", ")")
    if ts.accept("name", "bind"):
        ts.expect("op", "(")
        ts.expect("name", "c")
        cname = name
        if ts.accept("op", ","):
            ts.expect("name", "name")
            ts.expect("op", "=")
            cname = ts.expect("str")[1]
        ts.expect("op", ")")
        ts.bind_c = cname
    return kind, name, args, result, prefix_type


@dataclass
class CProc:
    """A procedure of an interface block with BIND(C): a function of a C library."""
    name: str
    cname: str
    kind: str
    args: list
    decls: dict
    result: VType | None
    where: str


def _read_c_interfaces(path, lines, i, consts, m):
    """Interface block without a generic name: BIND(C) procedures; returns the index of its END."""
    while True:
        no, text = lines[i]
        toks = tokenize(text)
        if toks[0] == ("name", "endinterface") or (toks[0] == ("name", "end") and len(toks) > 1
                                                   and toks[1] == ("name", "interface")):
            return i
        ts = Toks(toks, f"{path}:{no}")
        ts.bind_c = None
        hdr = _header(ts, consts)
        if hdr is None or ts.bind_c is None:
            raise FortranSubsetError(f"{path}:{no}: interface bodies other than BIND(C) procedures")
        kind, name, args, result, ptype = hdr
        decls = {}
        i += 1
        while True:
            bno, btext = lines[i]
            bt = tokenize(btext)
            if _is_end_of(bt, kind) or bt == [("name", "end")]:
                break
            if bt[0] == ("name", "import"):
                i += 1
                continue
            for v in parse_decl(Toks(bt, f"{path}:{bno}"), consts, f"{path}:{bno}"):
                decls[v.name] = v
            i += 1
        rtype = ptype
        if kind == "function" and rtype is None:
            rv = decls.get(result or name)
            rtype = rv.vt if rv is not None else None
        m.cprocs[name] = CProc(name, ts.bind_c, kind, args, decls, rtype, f"{path}:{no}")
        i += 1


def _is_end_of(text_toks, kind):
    t = text_toks
    if not t or t[0] != ("name", "end") and t[0] != ("name", "end" + kind):
        return False
    if t[0] == ("name", "end" + kind):
        return True
    return len(t) == 1 or t[1] == ("name", kind)


def read_module_file(path, consts) -> list[Module]:
    """Modules of a free-form source file, read at the specification level."""
    global _KINDS
    _KINDS = consts
    lines = logical_lines(path)
    mods = []
    i = 0
    while i < len(lines):
        no, text = lines[i]
        toks = tokenize(text)
        if toks[:1] == [("name", "module")] and len(toks) == 2:
            m, i = _read_module(path, lines, i, toks[1][1], consts)
            mods.append(m)
        elif toks[:1] == [("name", "program")] and len(toks) == 2:
            m, i = _read_program(path, lines, i, toks[1][1], consts)
            mods.append(m)
        else:
            i += 1
    return mods


def _read_program(path, lines, i, name, consts):
    """A main program as a module: its declarations become the module's variables (so a caller
    can read them after the run), its NAMELIST groups are recorded, and its executable part is
    the module's procedure `main`."""
    m = Module(name, str(path))
    m.is_program = True
    start_no = lines[i][0]
    i += 1
    while i < len(lines):
        no, text = lines[i]
        toks = tokenize(text)
        ts = Toks(toks, f"{path}:{no}")
        head = toks[0]
        if head == ("name", "use"):
            ts.next()
            mod = ts.expect("name")[1]
            only = None
            if ts.accept("op", ","):
                ts.expect("name", "only")
                ts.expect("op", ":")
                only = []
                while not ts.done():
                    only.append(ts.expect("name")[1])
                    ts.accept("op", ",")
            m.uses.append((mod, only, {}))
        elif head == ("name", "implicit"):
            pass
        elif head == ("name", "include"):
            m.includes.append(toks[1][1])
        elif head == ("name", "namelist"):
            ts.next()
            while not ts.done():
                ts.expect("op", "/")
                grp = ts.expect("name")[1]
                ts.expect("op", "/")
                names = []
                while ts.at("name"):
                    names.append(ts.next()[1])
                    if not ts.accept("op", ","):
                        break
                m.namelists[grp] = names
        elif _is_decl(ts):
            for v in parse_decl(ts, consts, f"{path}:{no}"):
                m.vars[v.name] = v
                if "parameter" in v.attrs and v.vt.base == "integer" and v.init is not None:
                    try:
                        consts[v.name] = _const_int(v.init, consts)
                    except FortranSubsetError:
                        pass
        else:
            break
        i += 1
    body = []
    while i < len(lines):
        no, text = lines[i]
        toks = tokenize(text)
        if toks[0] == ("name", "endprogram") or (toks[0] == ("name", "end") and
                                                 (len(toks) == 1 or toks[1] == ("name", "program"))):
            m.procs["main"] = ProcHeader("main", "subroutine", [], None, None, name, body, str(path),
                                         start_no)
            return m, i + 1
        if toks[0] == ("name", "contains"):
            raise FortranSubsetError(f"{path}:{no}: internal procedures of a program outside the subset")
        body.append((no, text))
        i += 1
    raise FortranSubsetError(f"{path}: program {name} not terminated")


def _read_module(path, lines, i, name, consts):
    m = Module(name, str(path))
    i += 1
    in_contains = False
    while i < len(lines):
        no, text = lines[i]
        where = f"{path}:{no}"
        toks = tokenize(text)
        ts = Toks(toks, where)
        head = toks[0] if toks else None
        if (head == ("name", "end") and len(toks) >= 2 and toks[1] == ("name", "module")) or \
                head == ("name", "endmodule") or (head == ("name", "end") and len(toks) == 1):
            return m, i + 1
        if in_contains:
            hdr = _header(ts, consts)
            if hdr is None:
                raise FortranSubsetError(f"{where}: expected a procedure in module {name}")
            kind, pname, args, result, ptype = hdr
            body = []
            i += 1
            depth = 0
            while True:
                if i >= len(lines):
                    raise FortranSubsetError(f"{where}: unterminated {kind} {pname}")
                bno, btext = lines[i]
                bt = tokenize(btext)
                if bt and bt[0] == ("name", "contains"):
                    raise FortranSubsetError(f"{path}:{bno}: internal procedures outside the subset")
                if _is_end_of(bt, kind) or (bt == [("name", "end")]):
                    break
                body.append((bno, btext))
                i += 1
            m.procs[pname] = ProcHeader(pname, kind, args, result, ptype, name, body, str(path), no)
            i += 1
            continue
        if head == ("name", "contains"):
            in_contains = True
        elif head == ("name", "use"):
            ts.next()
            mod = ts.expect("name")[1]
            only, renames = None, {}
            if ts.accept("op", ","):
                if ts.accept("name", "only"):
                    ts.expect("op", ":")
                    only = []
                    while not ts.done():
                        local = ts.expect("name")[1]
                        if ts.accept("op", "=>"):
                            remote = ts.expect("name")[1]
                            renames[local] = remote
                        only.append(local)
                        ts.accept("op", ",")
                else:
                    while not ts.done():
                        local = ts.expect("name")[1]
                        ts.expect("op", "=>")
                        renames[local] = ts.expect("name")[1]
                        ts.accept("op", ",")
            m.uses.append((mod, only, renames))
        elif head == ("name", "implicit"):
            pass
        elif head == ("name", "include"):
            m.includes.append(toks[1][1])
        elif head in (("name", "private"), ("name", "public")):
            ts.next()
            ts.accept("op", "::")
            names = []
            while not ts.done():
                names.append(ts.expect("name")[1])
                ts.accept("op", ",")
            if not names:
                m.default_private = head[1] == "private"
            else:
                (m.public if head[1] == "public" else m.private).update(names)
        elif head == ("name", "type") and not ts.at("op", "(", 1):
            ts.next()
            if ts.accept("op", ","):
                ts.expect("name")
                ts.accept("op", "::")
            ts.accept("op", "::")
            tname = ts.expect("name")[1]
            comps = {}
            i += 1
            while True:
                cno, ctext = lines[i]
                ct = tokenize(ctext)
                if ct[0] == ("name", "endtype") or (ct[0] == ("name", "end") and ct[1] == ("name", "type")):
                    break
                if ct[0] in (("name", "private"), ("name", "sequence")):
                    i += 1
                    continue
                for v in parse_decl(Toks(ct, f"{path}:{cno}"), consts, f"{path}:{cno}"):
                    comps[v.name] = v
                i += 1
            m.types[tname] = TypeDef(tname, comps)
        elif head == ("name", "interface"):
            ts.next()
            gname = ts.expect("name")[1] if not ts.done() else None
            if gname is None:
                i = _read_c_interfaces(path, lines, i + 1, consts, m) + 1
                continue
            specs = []
            i += 1
            while True:
                ino, itext = lines[i]
                it = tokenize(itext)
                if it[0] == ("name", "endinterface") or (it[0] == ("name", "end") and it[1] == ("name", "interface")):
                    break
                its = Toks(it, f"{path}:{ino}")
                its.expect("name", "module")
                its.expect("name", "procedure")
                while not its.done():
                    specs.append(its.expect("name")[1])
                    its.accept("op", ",")
                i += 1
            m.generics.setdefault(gname, []).extend(specs)
        elif _is_decl(ts):
            for v in parse_decl(ts, consts, where):
                m.vars[v.name] = v
                if "parameter" in v.attrs and v.vt.base == "integer" and v.init is not None:
                    try:
                        consts[v.name] = _const_int(v.init, consts)
                    except FortranSubsetError:
                        pass
        else:
            raise FortranSubsetError(f"{where}: statement outside the subset at module level: {text}")
        i += 1
    raise FortranSubsetError(f"{path}: module {name} not terminated")


def _const_int(e, consts):
    if e[0] == "int":
        return e[1]
    if e[0] == "name" and e[1] in consts:
        return consts[e[1]]
    if e[0] == "ref" and e[1] == ("name", "kind"):
        return _kind_value(e, consts)
    if e[0] == "un" and e[1] == "-":
        return -_const_int(e[2], consts)
    raise FortranSubsetError(f"non-constant integer parameter {e}")


# --------------------------------------------------------------------------- procedure bodies
@dataclass
class Proc:
    header: ProcHeader
    decls: dict          # name -> Var (dummies, locals, result)
    body: list           # statements
    uses: list
    formats: dict = field(default_factory=dict)   # FORMAT statements by label


class BodyParser:
    """Executable statements of one procedure into nested statement tuples:
      ('assign', lhs, rhs)  ('ptr', lhs, rhs)  ('call', name, args)
      ('if', [(cond, body)], else_body)  ('do', var, a, b, s, body)  ('while', cond, body)
      ('loop', body)  ('exit',)  ('cycle',)  ('return',)  ('stop',)  ('nop', text)
      ('alloc', [designators])  ('dealloc', [designators])  ('nullify', [designators])
      ('select', expr, [(cases, body)], default_body)
    """

    def __init__(self, header: ProcHeader, consts):
        self.h = header
        self.consts = consts
        self.lines = header.lines
        self.i = 0
        self.formats = {}

    def where(self, no):
        return f"{self.h.path}:{no}"

    def parse(self, decls_only=False) -> Proc:
        global _KINDS
        _KINDS = self.consts
        decls, uses = {}, []
        while self.i < len(self.lines):
            no, text = self.lines[self.i]
            toks = tokenize(text)
            ts = Toks(toks, self.where(no))
            if toks[0] == ("name", "use"):
                ts.next()
                mod = ts.expect("name")[1]
                only = None
                if ts.accept("op", ","):
                    ts.expect("name", "only")
                    ts.expect("op", ":")
                    only = []
                    while not ts.done():
                        only.append(ts.expect("name")[1])
                        ts.accept("op", ",")
                uses.append((mod, only, {}))
            elif toks[0] == ("name", "implicit"):
                pass
            elif toks[0] in (("name", "intrinsic"), ("name", "external")):
                pass
            elif _is_decl(ts) and not self._looks_like_assignment(toks):
                for v in parse_decl(ts, self.consts, self.where(no)):
                    decls[v.name] = v
            else:
                break
            self.i += 1
        if decls_only:
            return Proc(self.h, decls, None, uses)
        body = self.block(())
        return Proc(self.h, decls, body, uses, self.formats)

    @staticmethod
    def _looks_like_assignment(toks):
        # 'real(x) = ...' never occurs; a declaration never has '=' before '::' at depth 0
        return False

    def block(self, terminators):
        out = []
        while self.i < len(self.lines):
            no, text = self.lines[self.i]
            toks = tokenize(text)
            if toks and toks[0][0] == "int":
                # a statement label: FORMAT statements are kept by label, other labels are dropped
                # (no GO TO is in the subset, so nothing can jump to them)
                label = int(toks[0][1])
                text = text.lstrip()[len(str(toks[0][1])):].lstrip()
                toks = toks[1:]
                if toks and toks[0] == ("name", "format"):
                    self.formats[label] = text[text.index("("):]
                    self.i += 1
                    out.append(("nop", text))
                    continue
            key = self._keyword(toks)
            if key in terminators:
                return out
            self.i += 1
            out.append(self.statement(no, text, toks, key))
        if terminators:
            raise FortranSubsetError(f"{self.h.path}: block not terminated in {self.h.name}")
        return out

    @staticmethod
    def _keyword(toks):
        if not toks or toks[0][0] != "name":
            return None
        w = toks[0][1]
        w2 = toks[1][1] if len(toks) > 1 and toks[1][0] == "name" else None
        if w in ("endif", "enddo", "endselect"):
            return w
        if w == "end" and w2 in ("if", "do", "select"):
            return "end" + w2
        if w == "else":
            return "elseif" if w2 == "if" else "else"
        if w == "elseif":
            return "elseif"
        if w == "case":
            return "case"
        return None

    def statement(self, no, text, toks, key):
        ts = Toks(toks, self.where(no))
        w = toks[0][1] if toks[0][0] == "name" else None
        nxt = toks[1] if len(toks) > 1 else ("eof", None)
        is_assign = self._assignment_shape(toks)
        if w == "if" and nxt == ("op", "(") and not is_assign:
            ts.next()
            ts.expect("op", "(")
            cond = parse_expr(ts)
            ts.expect("op", ")")
            if ts.accept("name", "then"):
                if not ts.done():
                    ts.fail("text after THEN")
                return self._if_block(cond)
            # logical IF: one statement
            rest = toks[ts.i:]
            return ("if", [(cond, [self.statement(no, text, rest, self._keyword(rest))])], [])
        if w == "do" and not is_assign:
            ts.next()
            if ts.done():
                body = self.block(("enddo",))
                self.i += 1
                return ("loop", body)
            if ts.accept("name", "while"):
                ts.expect("op", "(")
                cond = parse_expr(ts)
                ts.expect("op", ")")
                body = self.block(("enddo",))
                self.i += 1
                return ("while", cond, body)
            if ts.at("int"):
                ts.fail("labelled DO outside the subset")
            var = ts.expect("name")[1]
            ts.expect("op", "=")
            a = parse_expr(ts)
            ts.expect("op", ",")
            b = parse_expr(ts)
            s = None
            if ts.accept("op", ","):
                s = parse_expr(ts)
            body = self.block(("enddo",))
            self.i += 1
            return ("do", var, a, b, s, body)
        if w == "select" and nxt == ("name", "case") and not is_assign:
            ts.next()
            ts.next()
            ts.expect("op", "(")
            sel = parse_expr(ts)
            ts.expect("op", ")")
            cases, default = [], None
            while True:
                cno, ctext = self.lines[self.i]
                ct = tokenize(ctext)
                k = self._keyword(ct)
                if k == "endselect":
                    self.i += 1
                    break
                if k != "case":
                    raise FortranSubsetError(f"{self.where(cno)}: expected CASE")
                self.i += 1
                cts = Toks(ct, self.where(cno))
                cts.next()
                if cts.accept("name", "default"):
                    default = self.block(("case", "endselect"))
                    continue
                cts.expect("op", "(")
                sels = []
                while True:
                    if cts.accept("op", ":"):
                        sels.append(("range", None, parse_expr(cts)))
                    else:
                        lo = parse_expr(cts)
                        if cts.accept("op", ":"):
                            hi = None if cts.at("op", ")") or cts.at("op", ",") else parse_expr(cts)
                            sels.append(("range", lo, hi))
                        else:
                            sels.append(("val", lo))
                    if cts.accept("op", ")"):
                        break
                    cts.expect("op", ",")
                cases.append((sels, self.block(("case", "endselect"))))
            return ("select", sel, cases, default or [])
        if w in ("exit", "cycle") and len(toks) == 1:
            return (w,)
        if w == "return" and len(toks) == 1:
            return ("return",)
        if w == "stop" and not is_assign:
            return ("stop", text)
        if w == "continue" and len(toks) == 1:
            return ("nop", text)
        if w in ("print", "write", "read", "open", "close", "format", "flush", "rewind", "inquire") \
                and not is_assign:
            if w == "read":
                # READ(unit, NML=group): the group's values come from the caller
                ts.next()
                ts.expect("op", "(")
                depth, grp = 1, None
                while depth and not ts.done():
                    k, v = ts.next()
                    if k == "name" and v == "nml" and ts.accept("op", "="):
                        grp = ts.expect("name")[1]
                    elif k == "op" and v == "(":
                        depth += 1
                    elif k == "op" and v == ")":
                        depth -= 1
                if grp is None or not ts.done():
                    ts.fail("READ other than a NAMELIST read outside the subset")
                return ("nml", grp)
            if w == "write":
                return self._write(ts, text)
            if w in ("open", "close"):
                return self._open_close(w, ts, text)
            return ("nop", text)
        if w == "call" and not is_assign:
            ts.next()
            name = ts.expect("name")[1]
            args = []
            if ts.accept("op", "("):
                if not ts.at("op", ")"):
                    args.append(_arg(ts))
                    while ts.accept("op", ","):
                        args.append(_arg(ts))
                ts.expect("op", ")")
            if not ts.done():
                ts.fail("text after CALL")
            return ("call", name, args)
        if w in ("allocate", "deallocate", "nullify") and nxt == ("op", "(") and not is_assign:
            ts.next()
            ts.expect("op", "(")
            items = [_arg(ts)]
            while ts.accept("op", ","):
                items.append(_arg(ts))
            ts.expect("op", ")")
            items = [x for x in items if x[0] != "kw"]  # stat= is ignored
            return ({"allocate": "alloc", "deallocate": "dealloc", "nullify": "nullify"}[w], items)
        if w in ("where", "forall", "goto") or (w == "go" and nxt == ("name", "to")):
            ts.fail(f"{w.upper()} outside the subset")
        if is_assign:
            lhs = _postfix(ts, ("name", ts.expect("name")[1]))
            if ts.accept("op", "=>"):
                return ("ptr", lhs, parse_expr(ts))
            ts.expect("op", "=")
            rhs = parse_expr(ts)
            if not ts.done():
                ts.fail(f"unexpected {ts.peek()[1]!r} after assignment")
            return ("assign", lhs, rhs)
        ts.fail(f"statement outside the subset: {text}")

    @staticmethod
    def _write(ts, text):
        """WRITE(unit, fmt) items: ('write', unit, fmt, [items]) with fmt ('label', n), ('str', text),
        ('star',) for list-directed, or ('expr', e). A list it cannot read (implied DO) is output
        only: ('nop', text)."""
        save = ts.i
        try:
            ts.next()
            ts.expect("op", "(")
            unit, fmt = None, None
            pos = 0
            while True:
                key = None
                if ts.at("name") and ts.at("op", "=", 1):
                    key = ts.next()[1]
                    ts.next()
                if ts.accept("op", "*"):
                    e = ("star",)
                elif ts.at("int") and (key == "fmt" or (key is None and pos == 1)):
                    e = ("label", int(str(ts.next()[1]).partition("_")[0]))
                else:
                    e = parse_expr(ts)
                if key == "unit" or (key is None and pos == 0):
                    unit = e
                elif key == "fmt" or (key is None and pos == 1):
                    fmt = e if e[0] in ("star", "label") else (("str", e[1]) if e[0] == "str" else ("expr", e))
                pos += 1
                if ts.accept("op", ")"):
                    break
                ts.expect("op", ",")
            items = []
            while not ts.done():
                items.append(parse_expr(ts))
                if not ts.accept("op", ","):
                    break
            if not ts.done() or unit is None:
                raise FortranSubsetError("write list")
            return ("write", unit, fmt or ("star",), items)
        except FortranSubsetError:
            ts.i = save
            return ("nop", text)

    @staticmethod
    def _open_close(w, ts, text):
        """OPEN(unit=, file=, ...) -> ('open', unit, file); CLOSE(unit) -> ('close', unit): the
        caller may attach files to units; other specifiers (status, action, iostat) are ignored."""
        try:
            ts.next()
            ts.expect("op", "(")
            unit = file = None
            pos = 0
            while True:
                key = None
                if ts.at("name") and ts.at("op", "=", 1):
                    key = ts.next()[1]
                    ts.next()
                e = parse_expr(ts)
                if key == "unit" or (key is None and pos == 0):
                    unit = e
                elif key == "file":
                    file = e
                pos += 1
                if ts.accept("op", ")"):
                    break
                ts.expect("op", ",")
            return (w, unit, file) if w == "open" else ("close", unit)
        except FortranSubsetError:
            return ("nop", text)

    @staticmethod
    def _assignment_shape(toks):
        """True when the statement is `designator = expr` or `designator => expr`, a designator
        being name { (...) | %name }."""
        if not toks or toks[0][0] != "name":
            return False
        i, n = 1, len(toks)
        while i < n:
            kind, val = toks[i]
            if kind == "op" and val in ("=", "=>"):
                return True
            if kind == "op" and val == "(":
                depth = 1
                i += 1
                while i < n and depth:
                    k2, v2 = toks[i]
                    if k2 == "op" and v2 in ("(", "(/", "["):
                        depth += 1
                    elif k2 == "op" and v2 in (")", "/)", "]"):
                        depth -= 1
                    i += 1
                continue
            if kind == "op" and val == "%" and i + 1 < n and toks[i + 1][0] == "name":
                i += 2
                continue
            return False
        return False

    def _if_block(self, cond):
        arms = []
        body = self.block(("elseif", "else", "endif"))
        arms.append((cond, body))
        else_body = []
        while True:
            no, text = self.lines[self.i]
            toks = tokenize(text)
            k = self._keyword(toks)
            self.i += 1
            if k == "endif":
                return ("if", arms, else_body)
            if k == "else":
                else_body = self.block(("endif",))
                continue
            ts = Toks(toks, self.where(no))
            ts.next()
            if ts.at("name", "if"):
                ts.next()
            ts.expect("op", "(")
            c = parse_expr(ts)
            ts.expect("op", ")")
            ts.expect("name", "then")
            arms.append((c, self.block(("elseif", "else", "endif"))))

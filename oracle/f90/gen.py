"""Python code generation for the Fortran 90 subset (the oracle's source runner).

TEST INFRASTRUCTURE ONLY (see oracle/f90/__init__.py). Every needed procedure
of the parsed modules becomes one Python function; module variables live in
one namespace object per module; derived types become classes. Generation is
static: names are resolved through the Fortran scoping rules (local, host
module, use association with ONLY/renames and PUBLIC/PRIVATE), generic
interfaces are resolved by the types and ranks of the actual arguments,
integer division, integer powers and type conversion on assignment are
decided from the declared types. Whatever the generator cannot place raises
FortranSubsetError instead of guessing.
"""
from __future__ import annotations

from dataclasses import dataclass

from .lex import FortranSubsetError
from .parse import BodyParser, Module, Var, VType, read_module_file

# kind parameters of the intrinsic module iso_c_binding
C_KINDS = {"c_int": 4, "c_double": 8, "c_float": 4, "c_long": 8, "c_int32_t": 4, "c_int64_t": 8,
           "c_size_t": 8, "c_bool": 1, "c_char": 1}


def _iso_c_binding() -> Module:
    m = Module("iso_c_binding", "<intrinsic module>")
    for n, k in C_KINDS.items():
        m.vars[n] = Var(n, VType("integer", 4), None, {"parameter"}, init=("int", k))
    m.vars["c_null_ptr"] = Var("c_null_ptr", VType("cptr", 8), None, {"parameter"})
    return m


@dataclass(frozen=True)
class T:
    base: str          # 'real' 'integer' 'logical' 'character' 'type' 'none'
    kind: int = 0
    rank: int = 0
    tname: str = ""


T_INT = T("integer", 4)
T_REAL = T("real", 8)
T_LOG = T("logical", 4)
T_STR = T("character", 1)
T_NONE = T("none")


def vt_t(vt: VType, rank: int) -> T:
    return T(vt.base, vt.kind, rank, vt.tname)


@dataclass
class Sym:
    cat: str            # local modvar saved proc generic type intrinsic host param
    var: Var = None
    code: str = ""      # python expression of the variable (FArr, object or scalar)
    lbs: tuple = None   # per-dimension lower-bound code, None where dynamic
    cache: str = ""     # python name bound to the variable's numpy data (fixed-shape arrays)
    owner: str = ""
    specs: list = None  # generic: [(module, proc name)]
    tdef: object = None


INTRINSICS = {
    "abs", "sqrt", "exp", "log", "log10", "sin", "cos", "tan", "asin", "acos", "atan", "atan2",
    "sinh", "cosh", "tanh", "min", "max", "mod", "modulo", "sign", "real", "dble", "float", "int",
    "nint", "floor", "ceiling", "sum", "product", "maxval", "minval", "maxloc", "minloc", "size",
    "lbound", "ubound", "shape", "allocated", "associated", "present", "dot_product", "trim",
    "adjustl", "len_trim", "len", "huge", "tiny", "epsilon", "kind", "null", "count", "any", "all",
    "transpose", "merge", "dfloat", "c_loc", "c_associated",
}

# specific (double precision) names of generic intrinsics
ALIASES = {"dsqrt": "sqrt", "dabs": "abs", "dexp": "exp", "dlog": "log", "dlog10": "log10",
           "dsin": "sin", "dcos": "cos", "dtan": "tan", "dasin": "asin", "dacos": "acos",
           "datan": "atan", "datan2": "atan2", "dsinh": "sinh", "dcosh": "cosh", "dtanh": "tanh",
           "dsign": "sign", "dmax1": "max", "dmin1": "min", "dmod": "mod", "idint": "int",
           "idnint": "nint", "iabs": "abs", "max0": "max", "min0": "min"}
INTRINSICS |= set(ALIASES)

_LIBM = {"exp", "log", "log10", "sin", "cos", "tan", "asin", "acos", "atan", "sinh", "cosh", "tanh",
         "sqrt"}


class Program:
    """Parsed modules and the generator state."""

    def __init__(self, files, includes=None, host_procs=(), stubs=None, use_aliases=None):
        self.aliases = {k.lower(): v.lower() for k, v in (use_aliases or {}).items()}
        self.consts: dict = dict(C_KINDS)
        self.mods: dict = {"iso_c_binding": _iso_c_binding()}
        for f in files:
            for m in read_module_file(f, self.consts):
                self.mods[m.name] = m
        self.includes = includes or {}       # include file -> {name: python value}
        self.host_procs = set(host_procs)     # external procedures the harness provides
        self.stubs = stubs or (lambda mod, proc: False)
        self._parsed: dict = {}
        self._exports: dict = {}
        self._scopes: dict = {}
        self.queue: list = []
        self.done: dict = {}

    # ------------------------------------------------------------------ scoping
    def parsed(self, mod, name):
        key = (mod, name)
        if key not in self._parsed:
            h = self.mods[mod].procs[name]
            # a stubbed procedure needs only its interface
            self._parsed[key] = BodyParser(h, self.consts).parse(decls_only=bool(self.stubs(mod, name)))
        return self._parsed[key]

    def own_entities(self, mname):
        m = self.mods[mname]
        out = {}
        for n, v in m.vars.items():
            out[n] = ("var", mname, v)
        for n, t in m.types.items():
            out[n] = ("type", mname, t)
        for n, h in m.procs.items():
            out[n] = ("proc", mname, h)
        for n, specs in m.generics.items():
            out[n] = ("generic", [(mname, s) for s in specs])
        for n, cp in m.cprocs.items():
            out[n] = ("cproc", mname, cp)
        for inc in m.includes:
            if inc not in self.includes:
                raise FortranSubsetError(f"{m.path}: include '{inc}' has no stand-in")
            for n in self.includes[inc]:
                out[n] = ("inc", mname, inc)
        return out

    @staticmethod
    def _merge(out, name, ent):
        old = out.get(name)
        if old is None or old == ent:
            out[name] = ent
        elif old[0] == "generic" and ent[0] == "generic":
            out[name] = ("generic", old[1] + [s for s in ent[1] if s not in old[1]])
        elif old[0] == "generic" and ent[0] == "proc":
            spec = (ent[1], ent[2].name)
            if spec not in old[1]:
                out[name] = ("generic", old[1] + [spec])
        elif old[0] == "proc" and ent[0] == "generic":
            spec = (old[1], old[2].name)
            out[name] = ("generic", [spec] + [s for s in ent[1] if s != spec])
        else:
            out[name] = ("ambiguous", old, ent)

    def _use_names(self, uses, out):
        for (um, only, ren) in uses:
            um = self.aliases.get(um, um)
            if um not in self.mods:
                raise FortranSubsetError(f"module {um} was not read")
            ex = self.exports(um)
            if only is None:
                for n, e in ex.items():
                    self._merge(out, n, e)
                for local, remote in ren.items():
                    if remote in ex:
                        self._merge(out, local, ex[remote])
            else:
                for local in only:
                    remote = ren.get(local, local)
                    if remote in ex:
                        self._merge(out, local, ex[remote])
                    else:
                        raise FortranSubsetError(f"{remote} is not public in {um}")

    def exports(self, mname):
        if mname in self._exports:
            return self._exports[mname]
        m = self.mods[mname]
        allnames = {}
        self._use_names(m.uses, allnames)
        for n, e in self.own_entities(mname).items():
            if e[0] == "generic" and n in allnames and allnames[n][0] == "generic":
                self._merge(allnames, n, e)
            else:
                allnames[n] = e

        def public(n):
            if n in m.public:
                return True
            if n in m.private:
                return False
            return not m.default_private

        out = {n: e for n, e in allnames.items() if public(n)}
        self._exports[mname] = out
        return out

    def scope(self, mname):
        if mname not in self._scopes:
            out = {}
            self._use_names(self.mods[mname].uses, out)
            for n, e in self.own_entities(mname).items():
                if e[0] == "generic" and n in out and out[n][0] in ("generic", "proc"):
                    self._merge(out, n, e)
                else:
                    out[n] = e
            self._scopes[mname] = out
        return self._scopes[mname]

    def typedef(self, tname, mname):
        e = self.scope(mname).get(tname)
        if e and e[0] == "type":
            return e[1], e[2]
        for mn, m in self.mods.items():  # a component's type seen through its own module
            if tname in m.types:
                return mn, m.types[tname]
        raise FortranSubsetError(f"derived type {tname} not found from {mname}")

    # ------------------------------------------------------------------ entry
    def need(self, mod, name):
        key = (mod, name)
        if key not in self.done and key not in self.queue:
            self.queue.append(key)
        return f"P_{mod}__{name}"

    def generate(self, entry_points) -> str:
        for mod, name in entry_points:
            self.need(mod, name)
        funcs = []
        while self.queue:
            mod, name = self.queue.pop(0)
            self.done[(mod, name)] = True
            stub = self.stubs(mod, name)
            if stub == "raise":
                funcs.append(f"def P_{mod}__{name}(*args, **kw):\n"
                             f"    raise _rt.NotTranslated({mod + '::' + name!r})\n")
                continue
            if stub:
                funcs.append(f"def P_{mod}__{name}(*args, **kw):\n    return None\n")
                continue
            funcs.append(ProcGen(self, mod, self.parsed(mod, name)).emit())
        types = self._emit_types()
        inits = self._emit_module_inits()
        out = ["def _build(_rt, _host):",
               "    import numpy as _np",
               "    FArr = _rt.FArr; _NO = _rt.NO; NS = _rt.NS"]
        for line in types + inits:
            out.append("    " + line)
        for f in funcs:
            for line in f.splitlines():
                out.append("    " + line)
        out.append("    _mods = {%s}" % ", ".join(f"{m!r}: M_{m}" for m in self._mod_order()))
        out.append("    _procs = {%s}" % ", ".join(f"{k!r}: P_{k[0]}__{k[1]}" for k in self.done))
        out.append("    _types = {%s}" % ", ".join(
            f"{(mn, tn)!r}: T_{mn}__{tn}" for mn in self._mod_order() for tn in self.mods[mn].types))
        out.append("    return _mods, _procs, _types")
        return "\n".join(out) + "\n"

    def _mod_order(self):
        order, seen = [], set()

        def visit(mn):
            if mn in seen:
                return
            seen.add(mn)
            for (um, _, _) in self.mods[mn].uses:
                visit(self.aliases.get(um, um))
            order.append(mn)

        for mn in self.mods:
            visit(mn)
        return order

    def _emit_types(self):
        lines = []
        for mn in self._mod_order():
            for tn, td in self.mods[mn].types.items():
                lines.append(f"class T_{mn}__{tn}(_rt.Derived):")
                lines.append(f"    __slots__ = {tuple(td.comps)!r}")
                for cn, cv in td.comps.items():
                    if "pointer" in cv.attrs:
                        lines.append(f"    _ptr_{cn} = True")
                lines.append("    def __init__(self):")
                if not td.comps:
                    lines.append("        pass")
                for cn, cv in td.comps.items():
                    lines.append(f"        self.{cn} = {self._default(cv, mn, None)}")
        return lines

    def _default(self, v: Var, mname, gen):
        if "pointer" in v.attrs or "allocatable" in v.attrs:
            return "None"
        if v.shape:
            if any(d in (":", "*") or d[1] in ("*", ":") for d in v.shape):
                return "None"
            g = gen or ExprGen(self, mname, {})
            bounds = ", ".join(f"({g.ex(lo)[0]}, {g.ex(hi)[0]})" for lo, hi in v.shape)
            return f"FArr.alloc(({bounds},), {self.dtype(v.vt)})"
        if v.vt.base == "type":
            tm, _ = self.typedef(v.vt.tname, mname)
            return f"T_{tm}__{v.vt.tname}()"
        return {"real": "0.0", "integer": "0", "logical": "False", "character": "''",
                "cptr": "None"}[v.vt.base]

    @staticmethod
    def dtype(vt: VType):
        return {"real": "_np.float64", "integer": "_np.int64", "logical": "_np.bool_",
                "character": "object", "type": "object", "cptr": "object"}[vt.base]

    def _emit_module_inits(self):
        lines = []
        for mn in self._mod_order():
            m = self.mods[mn]
            lines.append(f"M_{mn} = NS()")
            g = ExprGen(self, mn, {})
            for inc in m.includes:
                for n, val in self.includes[inc].items():
                    lines.append(f"M_{mn}.{n} = {val!r}")
            for n, v in m.vars.items():
                if v.init is not None:
                    code, t = g.ex(v.init)
                    if v.shape and t.rank == 0:
                        code = f"{self._default(v, mn, g)}; M_{mn}.{n}.a[...] = {code}"
                        lines.append(f"M_{mn}.{n} = " + code)
                        continue
                    if v.shape:
                        code = f"FArr(_np.asarray({code}, dtype={self.dtype(v.vt)}))"
                    else:
                        code = g.convert(code, t, vt_t(v.vt, 0))
                    lines.append(f"M_{mn}.{n} = {code}")
                else:
                    lines.append(f"M_{mn}.{n} = {self._default(v, mn, g)}")
        return lines


class ExprGen:
    """Expression code generation in a scope (module scope plus the given local symbols)."""

    def __init__(self, prog: Program, mod: str, local_syms: dict, proc_uses=()):
        self.prog = prog
        self.mod = mod
        self.locals = local_syms
        self.scope = dict(prog.scope(mod))
        if proc_uses:
            prog._use_names(proc_uses, self.scope)
        self.tmp = 0

    def fresh(self, base="_t"):
        self.tmp += 1
        return f"{base}{self.tmp}"

    # ---------------------------------------------------------------- symbols
    def sym(self, name) -> Sym:
        if name in self.locals:
            return self.locals[name]
        e = self.scope.get(name)
        if e is None:
            if name in INTRINSICS:
                return Sym("intrinsic", owner=name)
            if name in self.prog.host_procs:
                return Sym("host", code=f"_host[{name!r}]", owner=name)
            raise FortranSubsetError(f"unresolved name '{name}' in module {self.mod}")
        kind = e[0]
        if kind == "var":
            _, owner, v = e
            return Sym("modvar", v, f"M_{owner}.{v.name}", self._static_lbs(v, f"M_{owner}.{v.name}"),
                       owner=owner)
        if kind == "inc":
            _, owner, inc = e
            val = self.prog.includes[inc][name]
            vt = VType("integer", 4) if isinstance(val, int) else VType("real", 8)
            return Sym("modvar", Var(name, vt, None, {"parameter"}), f"M_{owner}.{name}", owner=owner)
        if kind == "proc":
            return Sym("proc", owner=e[1], var=None, specs=[(e[1], e[2].name)])
        if kind == "generic":
            return Sym("generic", specs=e[1])
        if kind == "type":
            return Sym("type", owner=e[1], tdef=e[2])
        if kind == "cproc":
            return Sym("cproc", owner=e[1], tdef=e[2])
        if kind == "ambiguous":
            raise FortranSubsetError(f"'{name}' is ambiguous in module {self.mod}")
        raise FortranSubsetError(f"unknown entity kind {kind}")

    def _static_lbs(self, v: Var, code):
        if not v.shape:
            return None
        out = []
        for d in v.shape:
            if d in (":", "*") or d[1] == ":":
                out.append(None)
            else:
                lo = d[0]
                out.append(str(lo[1]) if lo[0] == "int" else None)
        return tuple(out)

    # ---------------------------------------------------------------- typing helpers
    def convert(self, code, src: T, dst: T):
        """Code converting a scalar value of type src for assignment to type dst."""
        if dst.base == "real" and src.base == "integer":
            code = f"float({code})"
        elif dst.base == "integer" and src.base == "real":
            code = f"int({code})"
        if dst.base == "real" and dst.kind == 4 and not (src.base == "real" and src.kind == 4):
            code = f"_rt.r4({code})"
        return code

    @staticmethod
    def promote(a: T, b: T) -> T:
        rank = max(a.rank, b.rank)
        if a.base == "real" or b.base == "real":
            kind = max(a.kind if a.base == "real" else 0, b.kind if b.base == "real" else 0)
            return T("real", kind, rank)
        return T(a.base, a.kind, rank)

    # ---------------------------------------------------------------- expressions
    def ex(self, e):
        """(python code, T) of an expression in value context."""
        k = e[0]
        if k == "int":
            return repr(e[1]), T_INT
        if k == "real":
            return repr(e[1]), T("real", e[2])
        if k == "str":
            return repr(e[1]), T_STR
        if k == "log":
            return repr(e[1]), T_LOG
        if k == "paren":
            c, t = self.ex(e[1])
            return f"({c})", t
        if k == "cons":
            parts = [self.ex(x) for x in e[1]]
            if not parts:
                return "_np.zeros(0)", T("real", 8, 1)
            t = parts[0][1]
            for _, pt in parts[1:]:
                t = self.promote(t, pt) if t.base in ("real", "integer") else t
            dt = {"real": "_np.float64", "integer": "_np.int64", "logical": "_np.bool_"}.get(t.base, "object")
            return f"_rt.cons([{', '.join(c for c, _ in parts)}], {dt})", T(t.base, t.kind, 1, t.tname)
        if k == "name":
            return self._name_value(e[1])
        if k == "comp":
            obj, _ = self.obj(e[1])
            v = self._comp_var(e)
            if v.shape:
                return f"{obj}.{e[2]}.a", vt_t(v.vt, len(v.shape))
            return f"{obj}.{e[2]}", vt_t(v.vt, 0)
        if k == "ref":
            return self._ref_value(e)
        if k == "un":
            c, t = self.ex(e[2])
            if e[1] == "-":
                return f"(-{c})", t
            if t.rank:
                return f"_np.logical_not({c})", t
            return f"(not {c})", T_LOG
        if k == "bin":
            return self._binop(e)
        if k == "sec":
            raise FortranSubsetError("section triplet outside an array reference")
        raise FortranSubsetError(f"expression kind {k} outside the subset")

    def _name_value(self, n):
        s = self.sym(n)
        if s.cat in ("local", "modvar", "saved"):
            v = s.var
            if v.shape:
                data = s.cache or f"{s.code}.a"
                return data, vt_t(v.vt, len(v.shape))
            return s.code, vt_t(v.vt, 0)
        if s.cat == "proc" or s.cat == "generic":
            raise FortranSubsetError(f"procedure {n} used as a value")
        raise FortranSubsetError(f"name {n} ({s.cat}) has no value")

    def _comp_var(self, e) -> Var:
        _, base, cname = e
        bt = self.type_of_obj(base)
        if bt.base != "type":
            raise FortranSubsetError(f"component {cname} of a non-derived value")
        _, td = self.prog.typedef(bt.tname, self.mod)
        if cname not in td.comps:
            raise FortranSubsetError(f"type {bt.tname} has no component {cname}")
        return td.comps[cname]

    def type_of_obj(self, e) -> T:
        """Declared type of a designator (rank of the whole entity)."""
        if e[0] == "name":
            s = self.sym(e[1])
            if s.var is None:
                raise FortranSubsetError(f"{e[1]} is not a variable")
            return vt_t(s.var.vt, s.var.rank)
        if e[0] == "comp":
            v = self._comp_var(e)
            return vt_t(v.vt, v.rank)
        if e[0] == "ref":
            bt = self.type_of_obj(e[1])
            nsec = sum(1 for a in e[2] if a[0] == "sec")
            return T(bt.base, bt.kind, nsec, bt.tname)
        raise FortranSubsetError(f"not a designator: {e}")

    def obj(self, e):
        """(code of the object, T) of a designator in object context: the FArr of a whole array,
        the instance of a derived-type scalar, the value of another scalar."""
        if e[0] == "name":
            s = self.sym(e[1])
            if s.var is None:
                raise FortranSubsetError(f"{e[1]} is not a variable")
            return s.code, vt_t(s.var.vt, s.var.rank)
        if e[0] == "comp":
            o, _ = self.obj(e[1])
            v = self._comp_var(e)
            return f"{o}.{e[2]}", vt_t(v.vt, v.rank)
        if e[0] == "ref":
            info = self._array_info(e[1])
            if info is None:
                raise FortranSubsetError(f"not an array designator: {e}")
            code, t = self._subscript(info, e[2])
            if t.rank:
                return f"FArr({code})", t
            return code, t
        raise FortranSubsetError(f"not a designator: {e}")

    def _array_info(self, base):
        """(object code, data code, Var, lower-bound codes) of an array designator base, or None."""
        if base[0] == "name":
            s = self.sym(base[1])
            if s.cat in ("local", "modvar", "saved") and s.var.shape:
                lbs = s.lbs or (None,) * len(s.var.shape)
                lbc = tuple(lb if lb is not None else f"{s.code}.lb[{d}]" for d, lb in enumerate(lbs))
                return s.code, (s.cache or f"{s.code}.a"), s.var, lbc
            return None
        if base[0] == "comp":
            v = self._comp_var(base)
            if not v.shape:
                return None
            o, _ = self.obj(base[1])
            code = f"{o}.{base[2]}"
            lbs = self._static_lbs(v, code)
            lbc = tuple(lb if lb is not None else f"{code}.lb[{d}]" for d, lb in enumerate(lbs))
            return code, f"{code}.a", v, lbc
        return None

    def _index(self, idx_code, lb):
        try:
            return str(int(idx_code) - int(lb))
        except ValueError:
            if lb == "1":
                return f"{idx_code} - 1"
            return f"{idx_code} - {lb}"

    def _subscript(self, info, args):
        ocode, data, v, lbc = info
        if len(args) != len(v.shape):
            raise FortranSubsetError(f"{v.name}: {len(args)} subscripts for rank {len(v.shape)}")
        parts, rank = [], 0
        for d, a in enumerate(args):
            lb = lbc[d]
            if a[0] == "sec":
                rank += 1
                lo, hi, st = a[1:]
                if st is None:
                    lo_c = "" if lo is None else self._index(self._int(lo), lb)
                    if hi is None:
                        hi_c = ""
                    else:
                        hi_c = f"max(0, {self._int(hi)} - {lb} + 1)"
                    parts.append(f"{lo_c}:{hi_c}")
                else:
                    lo_c = "None" if lo is None else self._int(lo)
                    hi_c = "None" if hi is None else self._int(hi)
                    parts.append(f"_rt.sl({lo_c}, {hi_c}, {self._int(st)}, {lb}, {data}.shape[{d}])")
            else:
                c, t = self.ex(a)
                if t.rank:
                    raise FortranSubsetError("vector subscripts outside the subset")
                parts.append(self._index(c, lb))
        return f"{data}[{', '.join(parts)}]", vt_t(v.vt, rank)

    def _int(self, e):
        c, t = self.ex(e)
        if t.base != "integer":
            raise FortranSubsetError("non-integer subscript")
        return c

    def _ref_value(self, e):
        _, base, args = e
        info = self._array_info(base)
        if info is not None:
            return self._subscript(info, args)
        if base[0] != "name":
            raise FortranSubsetError(f"call through a component: {e}")
        s = self.sym(base[1])
        if s.cat == "intrinsic":
            return self.intrinsic(base[1], args)
        if s.cat in ("proc", "generic"):
            mod, name, proc = self.resolve_call(base[1], s, args)
            res = self.result_var(mod, proc)
            code = f"{self.prog.need(mod, name)}({self.actuals(mod, proc, args)})"
            if res.shape:
                return f"{code}.a", vt_t(res.vt, len(res.shape))
            return code, vt_t(res.vt, 0)
        if s.cat == "cproc":
            code, rt_, refs = self.ccall(s.tdef, args)
            if refs:
                raise FortranSubsetError(f"{base[1]}: by-reference scalar arguments of a C function "
                                         "are written back only in `variable = f(...)` statements")
            return code, rt_
        if s.cat == "host":
            return f"{s.code}({', '.join(self.obj(a)[0] if self._is_designator(a) else self.ex(a)[0] for a in args)})", T_REAL
        if s.cat in ("local", "modvar", "saved") and s.var.vt.base == "character":
            raise FortranSubsetError("substrings outside the subset")
        raise FortranSubsetError(f"{base[1]} ({s.cat}) referenced with arguments")

    # ---------------------------------------------------------------- calls
    def result_var(self, mod, proc):
        h = proc.header
        rname = h.result or h.name
        v = proc.decls.get(rname)
        if v is None:
            if h.prefix_type is None:
                raise FortranSubsetError(f"function {h.name}: result type not declared")
            v = Var(rname, h.prefix_type)
        return v

    def resolve_call(self, name, s, args):
        """(module, specific name, parsed procedure) for a reference to name with args."""
        specs = s.specs
        if len(specs) == 1:
            mod, pname = specs[0]
            return mod, pname, self.prog.parsed(mod, pname)
        atypes = []
        for a in args:
            if a[0] == "kw":
                atypes.append((a[1], self._arg_type(a[2])))
            else:
                atypes.append((None, self._arg_type(a)))
        matches = []
        for mod, pname in specs:
            p = self.prog.parsed(mod, pname)
            if self._matches(p, atypes):
                matches.append((mod, pname, p))
        if len(matches) != 1:
            raise FortranSubsetError(
                f"generic {name}: {len(matches)} specifics match {[t for _, t in atypes]}")
        return matches[0]

    def _arg_type(self, a):
        if self._is_designator(a):
            return self.type_of_obj(a) if a[0] != "ref" or self._array_info(a[1]) else self.ex(a)[1]
        return self.ex(a)[1]

    @staticmethod
    def _compatible(dv: Var, t: T):
        if dv.vt.base != t.base:
            return False
        if t.base == "type" and dv.vt.tname != t.tname:
            return False
        if t.base == "real" and dv.vt.kind != t.kind and t.kind != 0:
            return False
        return (dv.rank == 0) == (t.rank == 0)

    def _matches(self, p, atypes):
        dummies = p.header.args
        pos = 0
        used = set()
        for kw, t in atypes:
            if kw is None:
                if pos >= len(dummies):
                    return False
                dn = dummies[pos]
                pos += 1
            else:
                if kw not in dummies:
                    return False
                dn = kw
            used.add(dn)
            dv = p.decls.get(dn)
            if dv is None or not self._compatible(dv, t):
                return False
        for dn in dummies:
            if dn not in used and "optional" not in p.decls[dn].attrs:
                return False
        return True

    @staticmethod
    def _is_designator(a):
        return a[0] in ("name", "comp") or (a[0] == "ref" and a[1][0] in ("name", "comp"))

    def _order_actuals(self, proc, args):
        dummies = proc.header.args if hasattr(proc, "header") else proc.args
        out = [None] * len(dummies)
        pos = 0
        for a in args:
            if a[0] == "kw":
                out[dummies.index(a[1])] = a[2]
            else:
                out[pos] = a
                pos += 1
        while out and out[-1] is None:
            out.pop()
        return out

    def actual(self, dv: Var, a):
        """Code of one actual argument for the dummy dv."""
        if a is None:
            return "None"
        if dv.rank or dv.vt.base == "type" or "pointer" in dv.attrs or "allocatable" in dv.attrs:
            if self._is_designator(a):
                code, t = self.obj(a)
                if dv.rank and not t.rank:
                    raise FortranSubsetError("array element passed to an array dummy")
                return code
            code, t = self.ex(a)
            return f"_rt.as_farr({code})" if dv.rank else code
        code, t = self.ex(a)
        return self.convert(code, t, vt_t(dv.vt, 0)) if t.base != dv.vt.base else code

    def actuals(self, mod, proc, args):
        ordered = self._order_actuals(proc, args)
        out = []
        for dn, a in zip(proc.header.args, ordered):
            out.append(self.actual(proc.decls[dn], a))
        return ", ".join(out)

    def ccall(self, cp, args):
        """(code, result T, [actual designators of by-reference scalars]) of a call of a BIND(C)
        procedure through the C library handed over as _host['__cdll__']."""
        ordered = self._order_actuals(cp, args)
        specs, refs = [], []
        for dn, a in zip(cp.args, ordered):
            dv = cp.decls[dn]
            b = dv.vt.base
            if dv.rank:
                kind = {("real", 8): "a8", ("integer", 4): "a4"}.get((b, dv.vt.kind))
                if kind is None:
                    raise FortranSubsetError(f"{cp.name}: C array argument of type {b}")
                code = self.obj(a)[0] if self._is_designator(a) else f"_rt.as_farr({self.ex(a)[0]})"
            elif "value" in dv.attrs:
                kind = {"integer": "i", "real": "d", "cptr": "p"}[b]
                code = self.ex(a)[0]
            else:
                kind = {"integer": "ri", "real": "rd", "cptr": "rp"}[b]
                code = self.ex(a)[0]
                refs.append(a)
            specs.append(f"({kind!r}, {code})")
        res = None
        rt_ = T_NONE
        if cp.kind == "function":
            res = {"integer": "i", "real": "d", "cptr": "p"}[cp.result.base]
            rt_ = vt_t(cp.result, 0)
        return f"_rt.ccall(_host, {cp.cname!r}, {res!r}, [{', '.join(specs)}])", rt_, refs

    # ---------------------------------------------------------------- operators
    def _binop(self, e):
        _, op, a, b = e
        ca, ta = self.ex(a)
        cb, tb = self.ex(b)
        rank = max(ta.rank, tb.rank)
        if op in ("+", "-", "*", "/"):
            t = self.promote(ta, tb)
            if t.base == "real" and ta.base == "real" and tb.base == "real" and ta.kind == 4 and tb.kind == 4:
                if a[0] == "real" and b[0] == "real":
                    return f"_rt.r4({ca} {op} {cb})", T("real", 4, rank)
                raise FortranSubsetError("single-precision arithmetic outside the subset")
            if op == "/" and ta.base == "integer" and tb.base == "integer":
                return (f"_rt.idiv_arr({ca}, {cb})" if rank else f"_rt.idiv({ca}, {cb})"), t
            return f"({ca} {op} {cb})", t
        if op == "**":
            if tb.base == "integer":
                if ta.base == "integer":
                    return f"_rt.ipow({ca}, {cb})", T_INT
                if tb.rank:
                    raise FortranSubsetError("array exponent")
                return (f"_rt.powi_arr({ca}, {cb})" if ta.rank else f"_rt.powi({ca}, {cb})"), ta
            t = self.promote(ta, tb)
            if rank:
                return f"_rt.vec(_rt.rpow)({ca}, {cb})", t
            return f"_rt.rpow({ca}, {cb})", t
        if op in ("==", "/=", "<", "<=", ">", ">="):
            pyop = {"==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">="}[op]
            if ta.base == "character":
                if op not in ("==", "/="):
                    raise FortranSubsetError("character ordering outside the subset")
                c = f"_rt.streq({ca}, {cb})"
                return (c if op == "==" else f"(not {c})"), T_LOG
            return f"({ca} {pyop} {cb})", T("logical", 4, rank)
        if op in ("and", "or"):
            if rank:
                return f"_np.logical_{op}({ca}, {cb})", T("logical", 4, rank)
            return f"({ca} {op} {cb})", T_LOG
        if op in ("eqv", "neqv"):
            return f"({ca} {'==' if op == 'eqv' else '!='} {cb})", T("logical", 4, rank)
        if op == "//":
            return f"({ca} + {cb})", T_STR
        raise FortranSubsetError(f"operator {op}")

    # ---------------------------------------------------------------- intrinsics
    def intrinsic(self, name, args):
        name = ALIASES.get(name, name)
        pos = [a for a in args if a[0] != "kw"]
        kw = {a[1]: a[2] for a in args if a[0] == "kw"}
        if name == "null":
            return "None", T_NONE
        if name in ("allocated", "associated"):
            code, _ = self.obj(pos[0])
            if len(pos) > 1:
                tc, _ = self.obj(pos[1])
                return f"({code} is {tc})", T_LOG
            return f"({code} is not None)", T_LOG
        if name == "present":
            code, _ = self.obj(pos[0])
            return f"({code} is not None)", T_LOG
        if name == "c_associated":
            return f"_rt.c_associated({self.ex(pos[0])[0]})", T_LOG
        if name == "c_loc":
            a = pos[0]
            if a[0] == "ref" and self._array_info(a[1]) is not None:
                code, t = self._subscript(self._array_info(a[1]), a[2])
                if t.rank:
                    raise FortranSubsetError("C_LOC of an array section")
                data, _, idx = code.partition("[")
                return f"_rt.elem_addr({data}, ({idx[:-1]},))", T("cptr", 8)
            code, t = self.obj(a)
            if not t.rank:
                raise FortranSubsetError("C_LOC of a scalar")
            return f"_rt.arr_addr({code})", T("cptr", 8)
        if name in ("size", "lbound", "ubound", "shape"):
            dim = pos[1] if len(pos) > 1 else kw.get("dim")
            if self._is_designator(pos[0]) and (pos[0][0] != "ref" or self._array_info(pos[0][1])):
                ocode, t = self.obj(pos[0])
                info = ocode
            else:
                c, t = self.ex(pos[0])
                info = f"_rt.as_farr({c})"
            if name == "size":
                if dim is None:
                    return f"{info}.a.size", T_INT
                return f"{info}.a.shape[{self._int(dim)} - 1]", T_INT
            if name == "shape":
                return f"_np.array({info}.a.shape, dtype=_np.int64)", T("integer", 4, 1)
            if dim is None:
                raise FortranSubsetError(f"{name} without DIM")
            d = f"{self._int(dim)} - 1"
            if name == "lbound":
                return f"{info}.lb[{d}]", T_INT
            return f"({info}.lb[{d}] + {info}.a.shape[{d}] - 1)", T_INT
        vals = [self.ex(a) for a in pos]
        c = [v[0] for v in vals]
        t = [v[1] for v in vals]
        if name in _LIBM:
            if t[0].base == "integer":
                raise FortranSubsetError(f"{name} of an integer")
            if t[0].rank:
                if name == "sqrt":
                    return f"_np.sqrt({c[0]})", t[0]
                return f"_rt.vec(_rt.{name})({c[0]})", t[0]
            return f"_rt.{name}({c[0]})", t[0]
        if name == "atan2":
            if t[0].rank or t[1].rank:
                return f"_rt.vec(_rt.atan2)({c[0]}, {c[1]})", self.promote(t[0], t[1])
            return f"_rt.atan2({c[0]}, {c[1]})", self.promote(t[0], t[1])
        if name == "abs":
            return (f"_np.abs({c[0]})" if t[0].rank else f"abs({c[0]})"), t[0]
        if name in ("min", "max"):
            rt_ = t[0]
            for x in t[1:]:
                rt_ = self.promote(rt_, x)
            if rt_.rank:
                fn = "_np.minimum" if name == "min" else "_np.maximum"
                code = c[0]
                for x in c[1:]:
                    code = f"{fn}({code}, {x})"
                return code, rt_
            conv = [self.convert(ci, ti, T(rt_.base, rt_.kind)) for ci, ti in zip(c, t)]
            return f"{name}({', '.join(conv)})", rt_
        if name == "mod":
            if t[0].base == "integer":
                return f"_rt.imod({c[0]}, {c[1]})", T_INT
            return f"_rt.fmod({c[0]}, {c[1]})", t[0]
        if name == "modulo":
            if t[0].base == "integer":
                return f"({c[0]} % {c[1]})", T_INT
            return f"_rt.fmodulo({c[0]}, {c[1]})", t[0]
        if name == "sign":
            return f"_rt.sign({c[0]}, {c[1]})", t[0]
        if name in ("real", "dble", "float", "dfloat"):
            kind = 8 if name in ("dble", "dfloat") else 4
            if name == "real":
                k = kw.get("kind") or (pos[1] if len(pos) > 1 else None)
                if k is not None:
                    kind = self.prog.consts.get(k[1], None) if k[0] == "name" else (k[1] if k[0] == "int" else None)
                    if kind is None:
                        raise FortranSubsetError("REAL kind selector")
                elif t[0].base == "real":
                    kind = t[0].kind
            if t[0].rank:
                code = f"_np.asarray({c[0]}, dtype=_np.float64)"
                return (code if kind == 8 else f"_rt.r4({code})"), T("real", kind, t[0].rank)
            code = f"float({c[0]})"
            return (code if kind == 8 else f"_rt.r4({code})"), T("real", kind)
        if name == "int":
            if t[0].rank:
                return f"_np.trunc({c[0]}).astype(_np.int64)", T("integer", 4, t[0].rank)
            return f"int({c[0]})", T_INT
        if name == "nint":
            return f"_rt.nint({c[0]})", T_INT
        if name == "floor":
            return f"_rt.floor({c[0]})", T_INT
        if name == "ceiling":
            return f"_rt.ceil({c[0]})", T_INT
        if name == "sum":
            if len(pos) > 1 or kw:
                raise FortranSubsetError("SUM with DIM or MASK")
            if t[0].base == "integer":
                return f"_rt.isum({c[0]})", T_INT
            return f"_rt.fsum({c[0]})", T(t[0].base, t[0].kind)
        if name == "product":
            return f"_rt.fprod({c[0]})", T(t[0].base, t[0].kind)
        if name in ("maxval", "minval"):
            return f"_rt.{name}({c[0]})", T(t[0].base, t[0].kind)
        if name in ("maxloc", "minloc"):
            return f"_rt.{name}({c[0]})", T("integer", 4, 1)
        if name == "dot_product":
            return f"_rt.dot({c[0]}, {c[1]})", T(self.promote(t[0], t[1]).base, 8)
        if name == "trim":
            return f"{c[0]}.rstrip()", T_STR
        if name == "adjustl":
            return f"({c[0]}.lstrip() + ' ' * (len({c[0]}) - len({c[0]}.lstrip())))", T_STR
        if name == "len_trim":
            return f"len({c[0]}.rstrip())", T_INT
        if name == "len":
            return f"len({c[0]})", T_INT
        if name == "huge":
            return ("1.7976931348623157e308" if t[0].base == "real" else "2147483647"), T(t[0].base, t[0].kind)
        if name == "tiny":
            return "2.2250738585072014e-308", T_REAL
        if name == "epsilon":
            return ("2.220446049250313e-16" if t[0].kind == 8 else "1.1920928955078125e-07"), T("real", t[0].kind)
        if name == "kind":
            return str(t[0].kind), T_INT
        if name == "count":
            return f"int(_np.count_nonzero({c[0]}))", T_INT
        if name in ("any", "all"):
            return f"bool(_np.{name}({c[0]}))", T_LOG
        if name == "transpose":
            return f"_np.asfortranarray(_np.transpose({c[0]}))", t[0]
        if name == "merge":
            return f"({c[0]} if {c[2]} else {c[1]})", t[0]
        raise FortranSubsetError(f"intrinsic {name} outside the subset")


class ProcGen:
    """One procedure as a Python function."""

    def __init__(self, prog: Program, mod: str, proc):
        self.prog = prog
        self.mod = mod
        self.p = proc
        self.h = proc.header
        self.fname = f"P_{mod}__{self.h.name}"
        self.is_func = self.h.kind == "function"
        self.rname = (self.h.result or self.h.name) if self.is_func else None
        syms = {}
        self.saved = []
        for n, v in proc.decls.items():
            if n in self.h.args:
                syms[n] = self._local_sym(n, v, dummy=True)
            elif "save" in v.attrs or (v.init is not None and "parameter" not in v.attrs):
                code = f"S_{mod}__{self.h.name}.{n}"
                syms[n] = Sym("saved", v, code, self._lbs(v, dummy=False), owner=mod)
                self.saved.append(v)
            else:
                syms[n] = self._local_sym(n, v, dummy=False)
        if self.is_func and self.rname not in syms:
            v = Var(self.rname, self.h.prefix_type)
            proc.decls[self.rname] = v
            syms[self.rname] = self._local_sym(self.rname, v, dummy=False)
        self.g = ExprGen(prog, mod, syms, proc.uses)
        self.lines: list[str] = []
        self.ind = 1

    def _lbs(self, v: Var, dummy: bool):
        if not v.shape:
            return None
        out = []
        for d in v.shape:
            if d == ":":
                out.append("1" if dummy and not ({"pointer", "allocatable"} & v.attrs) else None)
            elif d == "*":
                out.append("1")
            elif d[1] == ":":  # assumed shape with a declared lower bound
                lo = d[0]
                out.append(str(lo[1]) if lo[0] == "int" else None)
            else:
                lo = d[0]
                out.append(str(lo[1]) if lo[0] == "int" else None)
        return tuple(out)

    def _local_sym(self, n, v: Var, dummy: bool):
        cache = ""
        if v.shape and not ({"pointer", "allocatable"} & v.attrs) and not (dummy and "optional" in v.attrs):
            cache = f"A_{n}"
        return Sym("local", v, f"v_{n}", self._lbs(v, dummy), cache)

    def w(self, s):
        self.lines.append("    " * self.ind + s)

    # ------------------------------------------------------------------ emission
    def writable(self):
        out = []
        for n in self.h.args:
            v = self.p.decls[n]
            wr = ({"pointer", "allocatable"} & v.attrs) or (
                v.rank == 0 and v.vt.base != "type" and v.intent != "in")
            out.append(bool(wr))
        return out

    def emit(self):
        args = []
        for n in self.h.args:
            v = self.p.decls.get(n)
            if v is None:
                raise FortranSubsetError(f"{self.h.path}:{self.h.lineno}: dummy {n} not declared")
            args.append(f"v_{n}=None" if "optional" in v.attrs else f"v_{n}")
        head = f"def {self.fname}({', '.join(args)}):"
        pre = []
        if self.saved:
            pre.append(f"S_{self.mod}__{self.h.name} = NS()")
            for v in self.saved:
                if v.init is not None:
                    code, t = self.g.ex(v.init)
                    pre.append(f"S_{self.mod}__{self.h.name}.{v.name} = {self.g.convert(code, t, vt_t(v.vt, 0))}")
                else:
                    pre.append(f"S_{self.mod}__{self.h.name}.{v.name} = {self.prog._default(v, self.mod, self.g)}")
        self.lines.append(head)
        # dummies: explicit-shape association, cached data
        for n in self.h.args:
            v = self.p.decls[n]
            s = self.g.locals[n]
            if v.shape and all(d != ":" and (d == "*" or d[1] != ":") for d in v.shape) and \
                    not ({"pointer", "allocatable"} & v.attrs):
                if any(d == "*" or d[1] == "*" for d in v.shape):
                    if len(v.shape) != 1:
                        raise FortranSubsetError("assumed-size arrays of rank > 1")
                    self.w(f"v_{n} = _rt.as_farr(v_{n}) if v_{n} is not None else None")
                else:
                    ext = ", ".join(f"({self.g._int(hi)}) - ({self.g._int(lo)}) + 1" for lo, hi in v.shape)
                    self.w(f"v_{n} = _rt.assoc(v_{n}, ({ext},))")
            if s.cache:
                self.w(f"{s.cache} = v_{n}.a")
        # locals
        for n, v in self.p.decls.items():
            if n in self.h.args or self.g.locals[n].cat != "local":
                continue
            if "parameter" in v.attrs:
                code, t = self.g.ex(v.init)
                if v.shape:
                    self.w(f"v_{n} = FArr(_np.asarray({code}, dtype={self.prog.dtype(v.vt)}))")
                else:
                    self.w(f"v_{n} = {self.g.convert(code, t, vt_t(v.vt, 0))}")
            else:
                self.w(f"v_{n} = {self.prog._default(v, self.mod, self.g)}")
            s = self.g.locals[n]
            if s.cache:
                self.w(f"{s.cache} = v_{n}.a")
        self.block(self.p.body)
        self.w(self._return())
        return "\n".join(pre + self.lines) + "\n"

    def _return(self):
        if self.is_func:
            return f"return v_{self.rname}"
        wr = self.writable()
        if not any(wr):
            return "return None"
        return "return (" + "".join(
            (f"v_{n}, " if w else "_NO, ") for n, w in zip(self.h.args, wr)) + ")"

    def block(self, stmts):
        if not stmts:
            self.w("pass")
        for s in stmts:
            self.stmt(s)

    def stmt(self, s):
        k = s[0]
        g = self.g
        if k == "assign":
            self.assign(s[1], s[2])
        elif k == "ptr":
            tgt, _ = g.obj(s[1]) if s[1][0] != "ref" else (None, None)
            if tgt is None:
                raise FortranSubsetError("pointer assignment to a section")
            if s[2][0] == "ref" and s[2][1] == ("name", "null"):
                self.w(f"{tgt} = None")
            else:
                src, _ = g.obj(s[2])
                self.w(f"{tgt} = {src}")
        elif k == "call":
            self.call(s[1], s[2])
        elif k == "if":
            first = True
            for cond, body in s[1]:
                c, _ = g.ex(cond)
                self.w(f"{'if' if first else 'elif'} {c}:")
                first = False
                self.ind += 1
                self.block(body)
                self.ind -= 1
            if s[2]:
                self.w("else:")
                self.ind += 1
                self.block(s[2])
                self.ind -= 1
        elif k == "do":
            _, var, a, b, st, body = s
            vs = g.sym(var)
            if vs.cat not in ("local", "modvar", "saved") or vs.var.rank or vs.var.vt.base != "integer":
                raise FortranSubsetError(f"DO variable {var} is not an integer scalar variable")
            lo, hi = g.fresh("_lo"), g.fresh("_hi")
            self.w(f"{lo} = {g._int(a)}; {hi} = {g._int(b)}")
            if st is None:
                self.w(f"for {vs.code} in range({lo}, {hi} + 1):")
                after = f"max({lo}, {hi} + 1)"
            else:
                stc = g.fresh("_st")
                self.w(f"{stc} = {g._int(st)}")
                self.w(f"for {vs.code} in _rt.do_range({lo}, {hi}, {stc}):")
                after = f"_rt.do_after({lo}, {hi}, {stc})"
            self.ind += 1
            self.block(body)
            self.ind -= 1
            self.w("else:")
            self.w(f"    {vs.code} = {after}")
        elif k == "while":
            c, _ = g.ex(s[1])
            self.w(f"while {c}:")
            self.ind += 1
            self.block(s[2])
            self.ind -= 1
        elif k == "loop":
            self.w("while True:")
            self.ind += 1
            self.block(s[1])
            self.ind -= 1
        elif k == "exit":
            self.w("break")
        elif k == "cycle":
            self.w("continue")
        elif k == "return":
            self.w(self._return())
        elif k == "stop":
            self.w(f"raise _rt.FortranStop({s[1]!r})")
        elif k == "nop":
            self.w("pass")
        elif k == "nml":
            grp = s[1]
            names = None
            for mn in [self.mod] + [u[0] for u in self.prog.mods[self.mod].uses]:
                names = self.prog.mods.get(mn) and self.prog.mods[mn].namelists.get(grp)
                if names:
                    break
            if not names:
                raise FortranSubsetError(f"namelist group {grp} not declared")
            nl = g.fresh("_nl")
            self.w(f"{nl} = _host['__namelist__'][{grp!r}]")
            for n in names:
                ts = g.sym(n)
                code = ts.code
                conv = {"integer": "int", "real": "float", "logical": "bool", "character": "str"}[ts.var.vt.base]
                self.w(f"if {n!r} in {nl}: {code} = {conv}({nl}[{n!r}])")
        elif k == "write":
            unit, fmt, items = s[1], s[2], s[3]
            if fmt[0] == "star":
                fcode = "None"
            elif fmt[0] == "label":
                if fmt[1] not in self.p.formats:
                    raise FortranSubsetError(f"{self.h.path}: FORMAT {fmt[1]} not found in {self.h.name}")
                fcode = repr(self.p.formats[fmt[1]])
            elif fmt[0] == "str":
                fcode = repr(fmt[1])
            else:
                fcode = g.ex(fmt[1])[0]
            try:
                vals = [g.ex(it)[0] for it in items]
            except FortranSubsetError:
                self.w("pass")
                return
            if unit[0] == "star":
                self.w(f"_rt.fwrite(_host, '*', {fcode}, [{', '.join(vals)}])")
                return
            uc, ut = g.ex(unit)
            if ut.base == "character":
                # internal write: the record becomes the variable's value; such strings only name
                # files and label log lines, so a format outside the formatter's subset leaves it
                r = g.fresh("_w")
                self.w(f"{r} = _rt.fformat_or_none({fcode}, [{', '.join(vals)}])")
                self.w(f"if {r} is not None:")
                self.ind += 1
                self.assign_code(unit, f"{r}[0]")
                self.ind -= 1
                return
            self.w(f"_rt.fwrite(_host, {uc}, {fcode}, [{', '.join(vals)}])")
        elif k in ("open", "close"):
            uc = g.ex(s[1])[0] if s[1] is not None else "None"
            if k == "open":
                fc = g.ex(s[2])[0] if s[2] is not None else "None"
                self.w(f"if '__open__' in _host: _host['__open__']({uc}, {fc})")
            else:
                self.w(f"if '__close__' in _host: _host['__close__']({uc})")
        elif k == "alloc":
            for item in s[1]:
                self.allocate(item)
        elif k in ("dealloc", "nullify"):
            for item in s[1]:
                code, _ = g.obj(item)
                self.w(f"{code} = None")
        elif k == "select":
            tmp = g.fresh("_sel")
            c, t = g.ex(s[1])
            self.w(f"{tmp} = {c}")
            first = True
            for sels, body in s[2]:
                conds = []
                for sel in sels:
                    if sel[0] == "val":
                        vc, _ = g.ex(sel[1])
                        conds.append(f"_rt.streq({tmp}, {vc})" if t.base == "character" else f"{tmp} == {vc}")
                    else:
                        parts = []
                        if sel[1] is not None:
                            parts.append(f"{tmp} >= {g.ex(sel[1])[0]}")
                        if sel[2] is not None:
                            parts.append(f"{tmp} <= {g.ex(sel[2])[0]}")
                        conds.append("(" + " and ".join(parts) + ")")
                self.w(f"{'if' if first else 'elif'} {' or '.join(conds)}:")
                first = False
                self.ind += 1
                self.block(body)
                self.ind -= 1
            if s[3]:
                self.w("else:" if not first else "if True:")
                self.ind += 1
                self.block(s[3])
                self.ind -= 1
        else:
            raise FortranSubsetError(f"statement {k}")

    def allocate(self, item):
        g = self.g
        if item[0] == "ref" and g.type_of_obj(item[1]).rank:
            base = item[1]
            code, t = g.obj(base)
            v = g.sym(base[1]).var if base[0] == "name" else g._comp_var(base)
            bounds = []
            for a in item[2]:
                if a[0] == "sec":
                    bounds.append(f"({g._int(a[1])}, {g._int(a[2])})")
                else:
                    bounds.append(f"(1, {g._int(a)})")
            self.w(f"{code} = FArr.alloc(({', '.join(bounds)},), {self.prog.dtype(v.vt)})")
            if v.vt.base == "type":
                tm, _ = self.prog.typedef(v.vt.tname, self.mod)
                self.w(f"for _i in range({code}.a.size): {code}.a.flat[_i] = T_{tm}__{v.vt.tname}()")
            return
        code, t = g.obj(item)
        if t.base != "type" or t.rank:
            raise FortranSubsetError(f"ALLOCATE of {item}")
        tm, _ = self.prog.typedef(t.tname, self.mod)
        self.w(f"{code} = T_{tm}__{t.tname}()")

    def assign(self, lhs, rhs):
        g = self.g
        if rhs[0] == "ref" and rhs[1][0] == "name" and g.sym(rhs[1][1]).cat == "cproc":
            code, rtype, refs = g.ccall(g.sym(rhs[1][1]).tdef, rhs[2])
            if refs:
                r = g.fresh("_c")
                self.w(f"{r} = {code}")
                for k, a in enumerate(refs):
                    self.assign_code(a, f"{r}[1][{k}]")
                self.assign_code(lhs, f"{r}[0]")
                return
        tt = g.type_of_obj(lhs)
        rc, rt_ = g.ex(rhs)
        if lhs[0] == "ref":
            info = g._array_info(lhs[1])
            if info is None:
                raise FortranSubsetError(f"assignment to {lhs}")
            code, t = g._subscript(info, lhs[2])
            if t.rank == 0:
                self.w(f"{code} = {g.convert(rc, rt_, t) if rt_.rank == 0 else rc}")
            else:
                self.w(f"{code} = {rc}")
            return
        code, t = g.obj(lhs)
        if t.rank:
            info = g._array_info(lhs)
            self.w(f"{info[1]}[...] = {rc}")
            return
        if t.base == "type":
            if rt_.base != "type":
                raise FortranSubsetError("derived-type assignment from another type")
            self.w(f"_rt.dcopy_into({code}, {rc})")
            return
        if rt_.rank:
            raise FortranSubsetError("array value assigned to a scalar")
        self.w(f"{code} = {g.convert(rc, rt_, t)}")

    def assign_code(self, lhs, code):
        """Assignment of a python value (a C result) to a scalar designator."""
        g = self.g
        if lhs[0] == "ref":
            tc, _ = g._subscript(g._array_info(lhs[1]), lhs[2])
        else:
            tc, _ = g.obj(lhs)
        self.w(f"{tc} = {code}")

    def call(self, name, args):
        g = self.g
        s = g.sym(name)
        if s.cat == "cproc":
            code, _, refs = g.ccall(s.tdef, args)
            r = g.fresh("_c")
            self.w(f"{r} = {code}")
            for k, a in enumerate(refs):
                self.assign_code(a, f"{r}[1][{k}]")
            return
        if s.cat == "host":
            parts, backs = [], []
            for k, a in enumerate(args):
                if a[0] == "kw":
                    raise FortranSubsetError("keyword argument to an external procedure")
                if g._is_designator(a):
                    code, t = g.obj(a)
                    parts.append(code)
                    base_sym = g.sym(a[1]) if a[0] == "name" else None
                    constant = base_sym is not None and (base_sym.var is None or
                                                         "parameter" in base_sym.var.attrs)
                    if not t.rank and t.base in ("integer", "real", "logical") and not constant:
                        backs.append((k, a))
                else:
                    parts.append(g.ex(a)[0])
            r = g.fresh("_h")
            self.w(f"{r} = {s.code}({', '.join(parts)})")
            if backs:
                # an external procedure may return one value per argument (_NO: unchanged)
                self.w(f"if {r} is not None:")
                self.ind += 1
                for k, a in backs:
                    self.w(f"if {r}[{k}] is not _NO:")
                    self.ind += 1
                    self.assign_code(a, f"{r}[{k}]")
                    self.ind -= 1
                self.ind -= 1
            return
        if s.cat not in ("proc", "generic"):
            raise FortranSubsetError(f"CALL of {name} ({s.cat})")
        mod, pname, proc = g.resolve_call(name, s, args)
        if proc.header.kind != "subroutine":
            raise FortranSubsetError(f"CALL of function {pname}")
        fn = self.prog.need(mod, pname)
        ordered = g._order_actuals(proc, args)
        callee = ProcGen.__new__(ProcGen)
        callee.p, callee.h = proc, proc.header
        wr = ProcGen.writable(callee)
        code = f"{fn}({g.actuals(mod, proc, args)})"
        backs = [(i, a) for i, (a, w) in enumerate(zip(ordered, wr)) if w and a is not None and g._is_designator(a)]
        if self.prog.stubs(mod, pname) or not backs:
            self.w(code)
            return
        r = g.fresh("_r")
        self.w(f"{r} = {code}")
        for i, a in backs:
            dv = proc.decls[proc.header.args[i]]
            if a[0] == "ref":
                info = g._array_info(a[1])
                tc, t = g._subscript(info, a[2])
                if t.rank:
                    continue  # a section passed to a pointer dummy keeps its data
            else:
                tc, t = g.obj(a)
                if t.rank and not ({"pointer", "allocatable"} & dv.attrs):
                    continue
            self.w(f"{tc} = {r}[{i}]")

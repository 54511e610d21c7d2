"""Run-time support of the Python code generated from the Fortran subset.

TEST INFRASTRUCTURE ONLY (see oracle/f90/__init__.py). Fortran REAL(8)
arithmetic is IEEE binary64 with every operation rounded once (no fused
multiply-add), which is what Python floats and numpy's element-wise operators
do; transcendental functions call the C library through Python's math module,
as compiled Fortran does. Arrays are numpy arrays in column-major order with
their lower bounds kept beside them (FArr).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np


class FortranStop(Exception):
    """A STOP statement was executed."""


class NotTranslated(Exception):
    """A procedure left out of the translation was called."""


class NS:
    """Namespace of one module's variables (or one procedure's saved locals)."""

    def __repr__(self):
        return f"NS({sorted(vars(self))})"


class Derived:
    """Base class of the generated derived types."""

    __slots__ = ()


class FArr:
    """A Fortran array: numpy data (column-major) and its lower bounds."""

    __slots__ = ("a", "lb")

    def __init__(self, a, lb=None):
        self.a = a
        self.lb = tuple(lb) if lb is not None else (1,) * a.ndim

    @staticmethod
    def alloc(bounds, dtype):
        ext = tuple(max(0, int(hi) - int(lo) + 1) for lo, hi in bounds)
        if dtype is object:
            a = np.empty(ext, dtype=object, order="F")
        else:
            a = np.zeros(ext, dtype=dtype, order="F")
        return FArr(a, tuple(int(lo) for lo, _ in bounds))

    def __repr__(self):
        return f"FArr(shape={self.a.shape}, lb={self.lb})"


NO = object()  # "no write-back" marker in a subroutine's returned tuple


def assoc(x, shape):
    """Explicit-shape dummy associated with an actual array (sequence association): the actual's
    elements in array-element order viewed with the dummy's shape."""
    if x is None:
        return None
    if not isinstance(x, FArr):
        x = FArr(np.asarray(x))
    if x.a.shape == tuple(shape):
        return x if x.lb == (1,) * len(shape) else FArr(x.a)
    n = int(np.prod(shape))
    flat = x.a.reshape(-1, order="F")
    if flat.size < n:
        raise ValueError(f"actual array of {flat.size} elements for a dummy of shape {shape}")
    v = flat[:n].reshape(shape, order="F")
    return FArr(v)


def as_farr(v):
    return v if isinstance(v, FArr) else FArr(np.asarray(v))


def sl(lo, hi, st, lb, ext):
    """Python slice of the Fortran triplet lo:hi:st on a dimension with lower bound lb and
    extent ext (lo/hi None = the bound)."""
    if lo is None:
        lo = lb if st > 0 else lb + ext - 1
    if hi is None:
        hi = lb + ext - 1 if st > 0 else lb
    a = lo - lb
    b = hi - lb
    if st > 0:
        return slice(a, b + 1 if b >= a else a, st)
    stop = b - 1
    return slice(a, stop if stop >= 0 else None, st) if b <= a else slice(a, a, st)


def do_range(a, b, s):
    if s == 0:
        raise ValueError("DO step 0")
    return range(a, b + 1, s) if s > 0 else range(a, b - 1, s)


def do_after(a, b, s):
    """Value of the DO variable after the loop completed (Fortran: start + trips * step)."""
    trips = max(0, (b - a + s) // s) if s > 0 else max(0, (a - b - s) // (-s))
    return a + trips * s


def idiv(a, b):
    """Integer division truncating toward zero."""
    a, b = int(a), int(b)
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def idiv_arr(a, b):
    return np.trunc(np.asarray(a, dtype=np.float64) / np.asarray(b, dtype=np.float64)).astype(np.int64)


def imod(a, p):
    a, p = int(a), int(p)
    return a - idiv(a, p) * p


def fmodulo(a, p):
    r = math.fmod(a, p)
    if r != 0.0 and ((r < 0.0) != (p < 0.0)):
        r += p
    return r


def powi(x, m):
    """x**m for integer m as GCC computes it (__powidf2: binary powering)."""
    m = int(m)
    n = -m if m < 0 else m
    y = x if n % 2 else 1.0
    while True:
        n >>= 1
        if not n:
            break
        x = x * x
        if n % 2:
            y = y * x
    return 1.0 / y if m < 0 else y


def powi_arr(x, m):
    return np.vectorize(lambda v: powi(float(v), m), otypes=[np.float64])(x)


def ipow(a, b):
    return int(a) ** int(b) if b >= 0 else idiv(1, int(a) ** (-int(b)))


def rpow(x, y):
    try:
        return math.pow(x, y)
    except (ValueError, OverflowError):
        return float("nan")


def _libm(fn):
    def f(*args):
        try:
            return fn(*args)
        except (ValueError, OverflowError):
            return float("nan")
    return f


sqrt = _libm(math.sqrt)
exp = _libm(math.exp)
log = _libm(math.log)
log10 = _libm(math.log10)
sin, cos, tan = math.sin, math.cos, math.tan
asin = _libm(math.asin)
acos = _libm(math.acos)
atan = math.atan
atan2 = math.atan2
sinh = _libm(math.sinh)
cosh = _libm(math.cosh)
tanh = math.tanh


def vec(fn):
    """Element-wise application of a scalar libm function to an array (same C library calls as
    the scalar case, rather than numpy's own vectorized implementations)."""
    def f(*args):
        return np.vectorize(lambda *v: fn(*(float(t) for t in v)), otypes=[np.float64])(*args)
    return f


fmod = math.fmod
floor = math.floor
ceil = math.ceil


def nint(x):
    r = math.floor(abs(x) + 0.5)
    return int(r) if x >= 0 else -int(r)


def sign(a, b):
    return abs(a) if b >= 0 else -abs(a)


def fsum(x):
    """SUM of an array: left-to-right in array-element order, as a compiler's strict loop."""
    s = 0.0
    for v in np.asarray(x).reshape(-1, order="F"):
        s = s + v
    return s


def isum(x):
    return int(np.asarray(x).sum())


def fprod(x):
    p = 1.0
    for v in np.asarray(x).reshape(-1, order="F"):
        p = p * v
    return p


def dot(a, b):
    a = np.asarray(a).reshape(-1, order="F")
    b = np.asarray(b).reshape(-1, order="F")
    s = 0.0
    for u, v in zip(a, b):
        s = s + u * v
    return s


def maxval(x):
    return np.asarray(x).max()


def minval(x):
    return np.asarray(x).min()


def maxloc(x):
    x = np.asarray(x)
    return np.array([int(np.argmax(x.reshape(-1, order="F"))) + 1], dtype=np.int64)


def minloc(x):
    x = np.asarray(x)
    return np.array([int(np.argmin(x.reshape(-1, order="F"))) + 1], dtype=np.int64)


def r4(x):
    """Rounding to a default-kind (binary32) REAL."""
    if isinstance(x, np.ndarray):
        return x.astype(np.float32).astype(np.float64)
    return float(np.float32(x))


def dcopy_into(dst, src):
    """Intrinsic assignment of a derived-type value: every component copied (pointer components
    keep their target)."""
    for k in dst.__slots__:
        v = getattr(src, k)
        if isinstance(v, FArr) and not getattr(type(dst), "_ptr_" + k, False):
            v = FArr(v.a.copy(order="F"), v.lb)
        setattr(dst, k, v)
    return dst


def streq(a, b):
    return a.rstrip() == b.rstrip()


def cons(parts, dtype):
    out = []
    for p in parts:
        if isinstance(p, np.ndarray):
            out.extend(p.reshape(-1, order="F").tolist())
        else:
            out.append(p)
    return np.array(out, dtype=dtype)


# --------------------------------------------------------------------------- iso_c_binding
def c_associated(p):
    return p is not None and p != 0


def arr_addr(x):
    return x.a.ctypes.data


def elem_addr(data, idx):
    return data.ctypes.data + sum(int(i) * st for i, st in zip(idx, data.strides))


_CTYPES = {"i": ctypes.c_int, "d": ctypes.c_double, "p": ctypes.c_void_p}


def ccall(host, cname, restype, args):
    """Call a BIND(C) procedure of the C library host['__cdll__']. args: (kind, value) with kind
    i/d/p by value, ri/rd/rp by reference (returned after the call), a8/a4 arrays of C double /
    C int passed as the address of their first element (a temporary copy, copied back, where
    the array is not contiguous or of another element type, as a compiler's copy-in/copy-out).
    Returns the result, or (result, [by-reference values]) when there are any."""
    f = getattr(host["__cdll__"], cname)
    f.restype = _CTYPES.get(restype) if restype else None
    cargs, refs, copies = [], [], []
    for kind, v in args:
        if kind in ("i", "d"):
            cargs.append(_CTYPES[kind](v))
        elif kind == "p":
            cargs.append(ctypes.c_void_p(v if v else None))
        elif kind in ("ri", "rd", "rp"):
            c = _CTYPES[kind[1]]() if v is None else _CTYPES[kind[1]](v)
            refs.append(c)
            cargs.append(ctypes.byref(c))
        elif kind in ("a8", "a4"):
            if v is None:
                cargs.append(ctypes.c_void_p(None))
                continue
            a = v.a if isinstance(v, FArr) else np.asarray(v)
            want = np.float64 if kind == "a8" else np.int32
            if a.dtype != want or not a.flags.f_contiguous:
                tmp = np.asfortranarray(a, dtype=want)
                copies.append((a, tmp))
                a = tmp
            cargs.append(ctypes.c_void_p(a.ctypes.data))
        else:
            raise ValueError(kind)
    r = f(*cargs)
    for a, tmp in copies:
        a[...] = tmp
    if not refs:
        return r
    return r, [c.value for c in refs]


# --------------------------------------------------------------------------- formatted output
def _parse_format(fmt: str):
    """A format specification '(...)' as nested nodes: ('lit', text), ('nl',), ('x', n),
    ('ed', repeat, letter, w, d), ('grp', repeat, [nodes])."""
    s = fmt.strip()
    if not (s.startswith("(") and s.endswith(")")):
        raise ValueError(f"format {fmt!r}")
    pos = 0

    def digits():
        nonlocal pos
        j = pos
        while pos < len(s) and s[pos].isdigit():
            pos += 1
        return int(s[j:pos]) if pos > j else None

    def group():
        nonlocal pos
        pos += 1
        out = []
        while True:
            while pos < len(s) and s[pos] in " ,:":
                pos += 1
            ch = s[pos]
            if ch == ")":
                pos += 1
                return out
            if ch in "'\"":
                j, text = pos + 1, []
                while True:
                    if s[j] == ch:
                        if j + 1 < len(s) and s[j + 1] == ch:
                            text.append(ch)
                            j += 2
                            continue
                        break
                    text.append(s[j])
                    j += 1
                out.append(("lit", "".join(text)))
                pos = j + 1
                continue
            if ch == "/":
                out.append(("nl",))
                pos += 1
                continue
            rep = digits()
            if s[pos] == "(":
                out.append(("grp", rep or 1, group()))
                continue
            j = pos
            while pos < len(s) and s[pos].isalpha():
                pos += 1
            letter = s[j:pos].upper()
            if letter == "X":
                out.append(("x", rep or 1))
                continue
            w = digits()
            d = None
            if pos < len(s) and s[pos] == ".":
                pos += 1
                d = digits()
            if letter not in ("A", "I", "F", "L"):
                raise NotImplementedError(f"edit descriptor {letter} outside the subset")
            out.append(("ed", rep or 1, letter, w, d))

    return group()


def _edit(letter, w, d, v):
    if letter == "A":
        t = str(v)
        if w is None:
            return t
        return t[:w] if len(t) >= w else " " * (w - len(t)) + t
    if letter == "L":
        t = "T" if v else "F"
        return t if w is None else t.rjust(w)
    if letter == "I":
        k = int(v)
        t = str(abs(k))
        if d is not None:
            t = t.zfill(d)
        if k < 0:
            t = "-" + t
        if not w:
            return t
        return t.rjust(w) if len(t) <= w else "*" * w
    if letter == "F":
        t = f"{float(v):.{d}f}"
        if not w:
            return t
        if len(t) > w and t.lstrip("-").startswith("0."):
            t = t.replace("0.", ".", 1)  # the optional leading zero goes first
        return t.rjust(w) if len(t) <= w else "*" * w
    raise NotImplementedError(letter)


def _flatten_items(items):
    out = []
    for v in items:
        if isinstance(v, np.ndarray):
            out.extend(v.reshape(-1, order="F").tolist())
        else:
            out.append(v)
    return out


def fformat(fmt, items):
    """Records written by a WRITE with format `fmt` (None: list-directed) of `items`. Formats use
    A, I, F, L, X, literals, '/' and repeated groups, with reversion to the last top-level group
    (the whole format when there is none); list-directed records are gfortran's layout for
    character and integer items (a leading blank, characters as they are, integers in 12
    columns)."""
    vals = _flatten_items(items)
    if fmt is None:
        parts = [" "]
        for v in vals:
            if isinstance(v, str):
                parts.append(v)
            elif isinstance(v, (int, np.integer)) and not isinstance(v, bool):
                parts.append(f"{int(v):12d}")
            else:
                raise NotImplementedError("list-directed output of non-character, non-integer items")
        return ["".join(parts)]
    nodes = _parse_format(fmt)
    records, cur = [], []
    k = 0

    def run(seq):
        nonlocal k
        for node in seq:
            kind = node[0]
            if kind == "lit":
                cur.append(node[1])
            elif kind == "x":
                cur.append(" " * node[1])
            elif kind == "nl":
                records.append("".join(cur))
                cur.clear()
            elif kind == "grp":
                for _ in range(node[1]):
                    if not run(node[2]):
                        return False
            else:
                _, rep, letter, w, d = node
                for _ in range(rep):
                    if k >= len(vals):
                        return False
                    cur.append(_edit(letter, w, d, vals[k]))
                    k += 1
        return True

    run(nodes)
    last_group = next((i for i in range(len(nodes) - 1, -1, -1) if nodes[i][0] == "grp"), None)
    restart = nodes[last_group:] if last_group is not None else nodes
    while k < len(vals):
        records.append("".join(cur))
        cur.clear()
        before = k
        run(restart)
        if k == before:
            raise ValueError(f"format {fmt!r} has no data edit descriptor for the remaining items")
    records.append("".join(cur))
    return records


def fformat_or_none(fmt, items):
    try:
        return fformat(fmt, items)
    except NotImplementedError:
        return None


def fwrite(host, unit, fmt, items):
    """WRITE to an external unit: the caller may collect the raw values (host['__write__']) and
    the formatted records (host['__record__'])."""
    if "__write__" in host:
        host["__write__"](unit, list(items))
    if "__record__" in host:
        host["__record__"](unit, fformat(fmt, items))

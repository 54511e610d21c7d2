"""Free-form Fortran 90 source reader and tokenizer for the subset runner.

TEST INFRASTRUCTURE ONLY (see oracle/f90/__init__.py). Turns a free-form
source file into logical statements (comments removed, `&` continuations
joined, `;` separated statements split) and a statement into tokens. Names are
lower-cased, since Fortran is case-insensitive; string literals keep their case.
"""
from __future__ import annotations

import re


class FortranSubsetError(Exception):
    """A construct outside the supported subset (the run stops rather than guess)."""


def _strip_comment(line: str) -> str:
    quote = None
    for i, ch in enumerate(line):
        if quote:
            if ch == quote:
                quote = None
        elif ch in "'\"":
            quote = ch
        elif ch == "!":
            return line[:i]
    return line


def _split_semicolons(s: str) -> list[str]:
    parts, quote, cur = [], None, []
    for ch in s:
        if quote:
            if ch == quote:
                quote = None
        elif ch in "'\"":
            quote = ch
        elif ch == ";":
            parts.append("".join(cur))
            cur = []
            continue
        cur.append(ch)
    parts.append("".join(cur))
    return [p for p in (q.strip() for q in parts) if p]


def logical_lines(path) -> list[tuple[int, str]]:
    """(first source line number, statement text) of every statement in the file."""
    with open(path, encoding="latin-1") as f:
        raw = f.read().splitlines()
    out: list[tuple[int, str]] = []
    buf, start = "", 0
    for no, line in enumerate(raw, 1):
        s = _strip_comment(line).strip()
        if not s:
            continue  # blank and comment lines do not end a continuation
        if buf:
            if s.startswith("&"):
                s = s[1:].lstrip()
            buf = buf + " " + s
        else:
            buf, start = s, no
        if buf.endswith("&"):
            buf = buf[:-1].rstrip()
            continue
        for part in _split_semicolons(buf):
            out.append((start, part))
        buf = ""
    if buf:
        raise FortranSubsetError(f"{path}: unterminated continuation at line {start}")
    return out


_DOTOPS = ("eqv", "neqv", "and", "or", "not", "eq", "ne", "lt", "le", "gt", "ge", "true", "false")
_DOT_RE = re.compile(r"\.(" + "|".join(_DOTOPS) + r")\.", re.I)
_REAL_RE = re.compile(
    r"(\d+\.\d*|\.\d+|\d+(?=[eEdD][+-]?\d))([eEdD][+-]?\d+)?(_[A-Za-z]\w*|_\d+)?")
_INT_RE = re.compile(r"\d+(_[A-Za-z]\w*|_\d+)?")
_NAME_RE = re.compile(r"[A-Za-z]\w*")
_OPS = ("**", "//", "==", "/=", "<=", ">=", "=>", "::", "(/", "/)",
        "<", ">", "=", "+", "-", "*", "/", "(", ")", ",", ":", "%", "[", "]")


def tokenize(s: str) -> list[tuple[str, object]]:
    """Tokens (kind, value): kinds 'name', 'int', 'real', 'str', 'op', 'dot' (dot operators and
    logical literals, value without dots)."""
    toks: list[tuple[str, object]] = []
    i, n = 0, len(s)
    while i < n:
        ch = s[i]
        if ch.isspace():
            i += 1
            continue
        if ch in "'\"":
            j = i + 1
            chars = []
            while True:
                if j >= n:
                    raise FortranSubsetError(f"unterminated string in: {s}")
                if s[j] == ch:
                    if j + 1 < n and s[j + 1] == ch:  # doubled quote
                        chars.append(ch)
                        j += 2
                        continue
                    break
                chars.append(s[j])
                j += 1
            toks.append(("str", "".join(chars)))
            i = j + 1
            continue
        if ch == ".":
            m = _DOT_RE.match(s, i)
            if m:
                toks.append(("dot", m.group(1).lower()))
                i = m.end()
                continue
        if ch.isdigit() or (ch == "." and i + 1 < n and s[i + 1].isdigit()):
            # an integer followed by a dot operator (1.eq.2) is not a real literal
            m_int = _INT_RE.match(s, i)
            if m_int and m_int.end() < n and s[m_int.end()] == "." and _DOT_RE.match(s, m_int.end()):
                m = None
            else:
                m = _REAL_RE.match(s, i)
            if m and (("." in m.group(0)) or m.group(2)):
                toks.append(("real", m.group(0)))
                i = m.end()
                continue
            m = _INT_RE.match(s, i)
            toks.append(("int", m.group(0)))
            i = m.end()
            continue
        if ch.isalpha():
            m = _NAME_RE.match(s, i)
            toks.append(("name", m.group(0).lower()))
            i = m.end()
            continue
        for op in _OPS:
            if s.startswith(op, i):
                # '(/' only opens an array constructor, never '(/=' or a division
                if op == "(/" and s.startswith("(/=", i):
                    continue
                toks.append(("op", op))
                i += len(op)
                break
        else:
            raise FortranSubsetError(f"unexpected character {ch!r} in: {s}")
    return toks

"""The FP32C visiting-order key (csrc/sphere_order.cuh): cube face by rank, 2-D Hilbert index on the
face. The face ranks and (u, v) orientations in the header must chain the six face curves into one
continuous curve (each face's curve ends at the cube corner where the next one starts); a numpy
replay of the key on an icosahedral grid then gives compact runs of targets. CPU only."""
import re
from pathlib import Path

import numpy as np

from thesiscode_b200 import grid

HEADER = Path(__file__).resolve().parents[1] / "thesiscode_b200" / "csrc" / "sphere_order.cuh"


def header_constants():
    text = HEADER.read_text()

    def const(name):
        m = re.search(name + r"\s*=\s*(0x[0-9a-fA-F]+|\d+)u?", text)
        assert m, name
        return int(m.group(1), 0)

    return (const("kFaceBits"), const("kFaceRank"), const("kFaceSwap"), const("kFaceFlipU"),
            const("kFaceFlipV"))


def face_of(x):
    ax = np.abs(x).argmax(1)
    major = x[np.arange(len(x)), ax]
    return 2 * ax + (major < 0), ax, major


def corner(face, U, V, swap, fu, fv):
    """3-D cube corner of curve coordinates (U, V) in {-1, 1} on `face`: the key maps face (u, v)
    to curve coordinates by swap, then reflections; this inverts it."""
    u, v = (-U if fu else U), (-V if fv else V)
    if swap:
        u, v = v, u
    a, s = face // 2, (-1 if face % 2 else 1)
    p = [0, 0, 0]
    others = [i for i in range(3) if i != a]
    p[a], p[others[0]], p[others[1]] = s, u, v
    return tuple(p)


def test_face_chain_is_continuous():
    _, rank, sw, fu, fv = header_constants()
    ranks = [(rank >> (3 * f)) & 7 for f in range(6)]
    assert sorted(ranks) == list(range(6))
    order = [ranks.index(r) for r in range(6)]
    o = {f: ((sw >> f) & 1, (fu >> f) & 1, (fv >> f) & 1) for f in range(6)}
    # the 2-D curve runs from cell (0, 0) to cell (n-1, 0): corners (-1,-1) -> (+1,-1)
    for f, g in zip(order, order[1:]):
        assert corner(f, 1, -1, *o[f]) == corner(g, -1, -1, *o[g]), (f, g)


def sphere_keys(x):
    """numpy replay of tcb::sphere_key."""
    bits, rank, sw, fu, fv = header_constants()
    face, ax, major = face_of(x)
    idx = np.arange(len(x))
    others = np.array([[1, 2], [0, 2], [0, 1]])[ax]
    u, v = x[idx, others[:, 0]], x[idx, others[:, 1]]
    s = ((sw >> face) & 1).astype(bool)
    u, v = np.where(s, v, u), np.where(s, u, v)
    u = np.where((fu >> face) & 1, -u, u)
    v = np.where((fv >> face) & 1, -v, v)
    n = 1 << bits
    X = np.clip(((u / np.abs(major) + 1) * 0.5 * n).astype(np.int64), 0, n - 1)
    Y = np.clip(((v / np.abs(major) + 1) * 0.5 * n).astype(np.int64), 0, n - 1)
    d = np.zeros(len(x), np.int64)
    q = n // 2
    while q > 0:
        rx, ry = (X & q) > 0, (Y & q) > 0
        d += q * q * ((3 * rx.astype(np.int64)) ^ ry.astype(np.int64))
        flip = ~ry & rx
        X, Y = np.where(flip, n - 1 - X, X), np.where(flip, n - 1 - Y, Y)
        X, Y = np.where(~ry, Y, X), np.where(~ry, X, Y)
        q //= 2
    return (((rank >> (3 * face)) & 7).astype(np.int64) << (2 * bits)) | d


def test_runs_of_keys_are_compact_patches():
    """Level 5 (20,480 panel centres): every run of 384 consecutive keys lies within 2.5x the
    radius of a disk holding 384 points (the patch radius bounds the FP32C offsets and the
    near-tile count)."""
    _, pans = grid.new_icos_grid(5)
    x = pans.x[~pans.hasChildren]
    order = np.argsort(sphere_keys(x), kind="stable")
    xs = x[order]
    tb = 384
    disk = np.sqrt(4 * tb / len(xs))
    worst = 0.0
    for b in range(0, len(xs), tb):
        t = xs[b:b + tb]
        c = t.mean(0)
        c /= np.linalg.norm(c)
        worst = max(worst, np.sqrt(((t - c) ** 2).sum(1).max()))
    assert worst <= 2.5 * disk, (worst, disk)

"""Regenerates the daligner2 bridging fixtures from the reference's own Handle_Redundancies.

daligner2 joins two paths of a pair that overlap narrowly in parallel (no common trace
point) through a fresh alignment of the overlap's box (DO_BRIDGING, dalign2/filter.c:1479-1705,
2124-2262).  No synthetic block makes that happen, so the cases are built at the level of one
pair: a read pair with a true overlap, its alignment from the oracle's Local_Alignment, and
two pieces of that alignment overlapping by a few trace intervals, the second shifted by a few
bases in B -- parallel, not entwined.  B-side paths come from the same alignment's B path.
Each case goes through oracle/_ref/d2_bridge_harness (the reference's Handle_Redundancies,
built from its sources by oracle/Makefile) and the outputs are stored beside the inputs.
Run from the repository root:

    make -C oracle ref liboracle.so && python tests/golden/make_d2_bridge_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import d2_bridge_cases as dbc  # noqa: E402
import oracle  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "d2_bridge_harness")
OUT = os.path.join(HERE, "d2_bridge", "cases.npz")
NCASES = 100


def mutate(rng, s, p_sub=0.03, p_ins=0.04, p_del=0.03):
    out = []
    for x in s:
        r = rng.random()
        if r < p_del:
            continue
        if r < p_del + p_sub:
            out.append((x + rng.integers(1, 4)) % 4)
        else:
            out.append(x)
        while rng.random() < p_ins:
            out.append(rng.integers(0, 4))
    return np.array(out, np.uint8)


def pieces(path, trace, tspace, i0, i1, shift):
    """The path over its trace intervals [i0, i1), B coordinates shifted."""
    abpos, bbpos, aepos, bepos, diffs, tlen = path
    nint = tlen // 2
    a0 = abpos // tspace

    def a_at(i):
        return abpos if i == 0 else (aepos if i >= nint else (a0 + i) * tspace)

    def b_at(i):
        return bbpos + int(trace[1:2 * i:2].sum())
    t = trace[2 * i0:2 * i1]
    return ([a_at(i0), b_at(i0) + shift, a_at(i1), b_at(i1) + shift, int(t[0::2].sum()), int(t.size)],
            t.astype(np.uint16))


def make_case(rng):
    tspace = int(rng.choice([100, 100, 100, 200]))
    comp = int(rng.integers(0, 2))
    has_b = int(rng.integers(0, 2))
    la = int(rng.integers(2500, 4500))
    a = rng.integers(0, 4, la).astype(np.uint8)
    s0 = int(rng.integers(200, 600))
    s1 = la - int(rng.integers(200, 600))
    m = mutate(rng, a[s0:s1])
    fl = rng.integers(0, 4, int(rng.integers(200, 500))).astype(np.uint8)
    fr = rng.integers(0, 4, int(rng.integers(200, 500))).astype(np.uint8)
    b = np.concatenate([fl, m, fr])
    # a seed in the middle of the overlap: A position mid, B position by length ratio
    mid = (s0 + s1) // 2
    bp = fl.size + int((mid - s0) * m.size / (s1 - s0))
    p = oracle.make_params([.25] * 4, s=tspace)
    A4 = np.concatenate([[4], a, [4]]).astype(np.uint8)
    B4 = np.concatenate([[4], b, [4]]).astype(np.uint8)
    out, at, bt, _ = oracle.local_alignment(A4, B4, comp, mid - bp, mid + bp, p)
    apath, bpath = [int(x) for x in out[:6]], [int(x) for x in out[6:]]
    na, nb = apath[5] // 2, bpath[5] // 2
    if na < 10 or (has_b and nb < 10):
        return None
    amatch, bmatch = [], []

    def two(path, trace, n, store, swap=False):
        m1 = int(rng.integers(5, n - 3))
        m0 = m1 - int(rng.integers(1, 5))
        d = int(rng.choice([-4, -3, -2, -1, 1, 2, 3, 4]))
        p1 = pieces(path, trace, tspace, 0, m1, 0)
        p2 = pieces(path, trace, tspace, m0, n, d)
        store.extend([p2, p1] if swap else [p1, p2])
    two(apath, at, na, amatch)
    if has_b:
        # a complement pair's B path runs the other way: the A prefix's B side is the B
        # path's suffix; one case in five keeps the wrong order (the reference skips it)
        two(bpath, bt, nb, bmatch, swap=bool(comp) != (rng.random() < 0.2))
    # sometimes a third path: a copy of a piece (fused/contained) or a short unrelated piece
    if rng.random() < 0.3:
        i0 = int(rng.integers(0, na - 3))
        amatch.append(pieces(apath, at, tspace, i0, min(na, i0 + int(rng.integers(2, 6))), int(rng.integers(0, 3))))
        if has_b:
            j0 = int(rng.integers(0, nb - 3))
            bmatch.append(pieces(bpath, bt, tspace, j0, min(nb, j0 + int(rng.integers(2, 6))), 0))
    order = rng.permutation(len(amatch))
    amatch = [amatch[i] for i in order]
    if has_b:
        bmatch = [bmatch[i] for i in order]
    return dbc.Case(a, b, tspace, comp, amatch, bmatch if has_b else None)


def main():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    rng = np.random.default_rng(20241203)
    cases = []
    while len(cases) < NCASES:
        c = make_case(rng)
        if c is not None:
            cases.append(c)
    tmp = OUT + ".harness.bin"
    subprocess.run([HARNESS, tmp], input=b"".join(dbc.encode(c) for c in cases), stdout=subprocess.DEVNULL,
                   check=True)
    with open(tmp, "rb") as f:
        res = f.read()
    os.remove(tmp)
    expected = dbc.decode_results(res, cases)
    dbc.save(OUT, cases, expected)
    bridged = sum(1 for c, e in zip(cases, expected) if dbc.was_bridged(c, e))
    print(f"{len(cases)} cases, {bridged} with a bridge, written to {OUT}")


if __name__ == "__main__":
    main()

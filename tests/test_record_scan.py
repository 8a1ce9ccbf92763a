"""The aligner's record scan skip against the reference's sequential best-point loop.

forward_wave (dalign/align.c:880-897) visits a wave's diagonals in scan order; every new
maximum of the anti-diagonal c is a record, a record that passes PATH_AVE (q1) sets lasta, and
one that also passes the trim test (q2) sets the trim point.  The device (marvel_b200/csrc/
gd_align.cu, the best point of wave_step) takes the warp maximum, settles everything from its
first lane jm when jm passes both tests, and otherwise runs a prefix-max scan over the lanes
before jm only when a q1 lane precedes jm and that can matter: jm fails q1 (lasta), or a q2
lane precedes jm (the trim point).  This restates both on random waves, including the
adversarial ones where the skip would be wrong if the condition were weaker, and requires the
same besta, lasta and trim lane.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest


def reference(c, q1, q2, besta, lasta):
    trim = -1
    for i in range(len(c)):
        if c[i] > besta:
            besta = c[i]
            if q1[i]:
                lasta = c[i]
                if q2[i]:
                    trim = i
    return besta, lasta, trim


def device(c, q1, q2, besta, lasta):
    """The warp logic of one 32-lane chunk, forward direction (wv = c)."""
    n = len(c)
    wbest = besta
    Q1 = [q1[i] and c[i] > wbest for i in range(n)]  # the device's q1 includes wv > wbest
    Q2 = [Q1[i] and q2[i] for i in range(n)]
    wmax = max(c) if n else None
    trim = -1
    scans = 0
    if n and wmax > wbest:
        jm = c.index(wmax)
        mq1 = sum(1 << i for i in range(n) if Q1[i])
        mq2 = sum(1 << i for i in range(n) if Q2[i])
        besta = wmax
        p1j, p2j = (mq1 >> jm) & 1, (mq2 >> jm) & 1
        if p1j:
            lasta = besta
        if p2j:
            trim = jm
        else:
            before = (1 << jm) - 1
            if (mq1 & before) and (not p1j or (mq2 & before)):
                scans += 1
                excl, rec = -(1 << 62), []
                for i in range(n):
                    rec.append(c[i] > max(wbest, excl) and i < jm)
                    excl = max(excl, c[i])
                m1 = [i for i in range(n) if rec[i] and Q1[i]]
                if m1 and not p1j:
                    lasta = c[m1[-1]]
                m2 = [i for i in range(n) if rec[i] and Q2[i]]
                if m2:
                    trim = m2[-1]
    return besta, lasta, trim, scans


@pytest.mark.parametrize("seed", range(8))
def test_scan_skip_equals_sequential_records(seed):
    rng = np.random.default_rng(seed)
    scans = 0
    for _ in range(4000):
        n = int(rng.integers(1, 33))
        besta = int(rng.integers(0, 60))
        lasta = int(rng.integers(0, besta + 1))
        c = [int(x) for x in rng.integers(0, 80, n)]
        p = rng.random()
        q1 = [bool(x) for x in rng.random(n) < p]
        q2 = [bool(a and b) for a, b in zip(q1, rng.random(n) < rng.random())]
        want = reference(c, q1, q2, besta, lasta)
        got = device(c, q1, q2, besta, lasta)
        assert got[:3] == want, (c, q1, q2, besta, lasta, got, want)
        scans += got[3]
    assert scans > 0  # the random waves do reach the scan

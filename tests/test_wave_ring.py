"""The aligner's single wave ring against a ring per wave parity (CPU model of the reads).

marvel_b200/csrc/gd_align.cu updates one 128-diagonal ring per warp in place (wave_step):
the diagonals of a wave are processed in chunks of 32 lanes, every lane of a chunk reads its
predecessors (V at k+S, k, k-S inside the previous band; T/HA/HB at the chosen one; NA/NB at
k clamped to the previous band) before any lane of the chunk writes, and a chunk's first lane
takes what it reads from the previous chunk's last diagonal (its kP, and NA/NB when it is a new
band edge next to that chunk) from the edge that lane saved before writing.  This model runs
random band sequences (widening, minp/maxp clamps, WAVE_LAG-like trims, both directions, up to
four chunks) through both schemes and requires every lane to read the same values.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

RG, TW = 128, 32
NONE_F, NONE_R = -1, 1 << 30


def choose(FWD, k, vP, vC, vN):
    S = 1 if FWD else -1
    wP, wC, wN = (vP, vC, vN) if FWD else (-vP, -vC, -vN)
    if wC < wN:
        return (k + S) if wN < wP else (k - S)
    if wC < wP:
        return k + S
    return k


def wave_reads(FWD, olow, ohgh, low, hgh, rng_vals, two, ring, edge_store):
    """Reads of every lane; writes new values.  two: dict ring per parity (prev, cur) or None."""
    S = 1 if FWD else -1
    NONE = NONE_F if FWD else NONE_R
    width = hgh - low + 1
    nch = (width + TW - 1) // TW
    reads = []
    prev = two[0] if two is not None else ring
    cur = two[1] if two is not None else ring
    edges = {}
    for ch in range(nch):
        lanes = []
        for lane in range(TW):
            p = ch * TW + lane
            if p >= width:
                continue
            k = hgh - p if FWD else low + p
            kP, kN = k + S, k - S
            inb = lambda x: olow <= x <= ohgh
            vP = prev[x][0] if inb(x := kP) else NONE
            vC = prev[k][0] if inb(k) else NONE
            vN = prev[kN][0] if inb(kN) else NONE
            fromedge = two is None and ch > 0 and lane == 0
            if fromedge:
                vP = edges[ch - 1]["v"]
            ks = choose(FWD, k, vP, vC, vN)
            t, ha, hb = prev[ks][1], prev[ks][2], prev[ks][3]
            if fromedge and ks == kP:
                e = edges[ch - 1]
                t, ha, hb = e["t"], e["ha"], e["hb"]
            kn = min(max(k, olow), ohgh)
            na, nb = prev[kn][4], prev[kn][5]
            if fromedge and kn == kP:
                na, nb = edges[ch - 1]["na"], edges[ch - 1]["nb"]
            if two is None and lane == TW - 1 and ch + 1 < nch:
                edges[ch] = dict(v=vC, t=prev[k][1], ha=prev[k][2], hb=prev[k][3], na=na, nb=nb)
            lanes.append((k, (vP, vC, vN, ks, t, ha, hb, na, nb)))
        # every lane of the chunk has read: now the writes
        for k, r in lanes:
            reads.append((k, r))
            cur[k] = tuple(int(x) for x in rng_vals[k % len(rng_vals)])
    return reads


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("FWD", [True, False])
def test_single_ring_reads_what_two_rings_read(seed, FWD):
    rng = np.random.default_rng(seed * 2 + int(FWD))
    span = 4 * RG
    init = {k: tuple(int(x) for x in rng.integers(0, 1 << 20, 6)) for k in range(-span, span)}
    ring = dict(init)                    # the single ring (indexed by k; k & RM aliasing is not modelled)
    rings = [dict(init), dict(init)]     # [dif & 1]
    olow = ohgh = int(rng.integers(-20, 20))
    minp, maxp = -10 ** 9, 10 ** 9
    if rng.random() < 0.5:
        minp = olow - int(rng.integers(0, 40))
    for dif in range(1, 400):
        low, hgh = olow - 1, ohgh + 1
        if low < minp:
            low += 1
        if hgh > maxp:
            hgh -= 1
        if hgh - low + 1 > RG:
            break
        vals = rng.integers(0, 1 << 20, (RG + 8, 6))
        two = (rings[(dif - 1) & 1], rings[dif & 1])
        r2 = wave_reads(FWD, olow, ohgh, low, hgh, vals, two, None, None)
        r1 = wave_reads(FWD, olow, ohgh, low, hgh, vals, None, ring, None)
        assert r1 == r2, (dif, olow, ohgh, low, hgh)
        # the next band: grow most of the time (to reach several chunks), trim now and then
        u = rng.random()
        if u < 0.15 and hgh > low:
            a = int(rng.integers(low, hgh + 1))
            b = int(rng.integers(a, hgh + 1))
            olow, ohgh = a, b
        else:
            olow, ohgh = low, hgh

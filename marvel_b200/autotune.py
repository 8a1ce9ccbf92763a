"""Autotuner of the aligner's launch schedule, per read-length class.

The seed scan and alignment kernel (k_align_pairs) is nine tenths of a block comparison.
How its work is launched is a free choice -- every schedule gives the same records
(tests/test_gpu_parity.py) -- so this module times the choices on the blocks at hand and
keeps the fastest:

* the schedule: every pair group in one persistent launch, taken longest first from a
  device queue, or one launch per length class (classes of alen + blen, split at quantiles
  of the block's pair lengths);
* per length class, the kernel instance: a warp per alignment with 128-diagonal wave rings
  (4 warps per CTA, 6 CTAs per SM; a group whose band outgrows 128 diagonals is redone by the
  wide instance), the wide instance (512-diagonal rings, one warp per CTA), which takes such
  groups in one pass, or the duo instance (two 16-lane teams per warp, each on its own pair
  group with 128-diagonal rings), meant to keep twice the lanes busy on the narrow bands most
  waves have (it measures slower on every workload: the ring pairs halve the resident warps).

Candidates are timed on the loaded blocks (the aligner's device time of both orientations,
gd_stats.ms_align, best of `repeats` runs).  The radix sorts have no choice here: their
digit is 8 bits, the width the bulk-copy scatter's per-warp tables and digit runs are laid
out for.
"""
from __future__ import annotations

import numpy as np

from . import Context, run_loaded


def length_edges(A, B=None, nclasses=3):
    """alen + blen edges (bp) that split a block pair's read-pair lengths into nclasses
    classes of about equal work: quantiles of the sum of two random read lengths, weighted by
    length (an alignment's cost grows with its reads)."""
    la = np.asarray(A.rlen, np.float64)
    lb = la if B is None else np.asarray(B.rlen, np.float64)
    rng = np.random.default_rng(0)
    s = rng.choice(la, 20000) + rng.choice(lb, 20000)
    s.sort()
    w = np.cumsum(s) / s.sum()
    return sorted({int(s[np.searchsorted(w, q)]) for q in np.linspace(0, 1, nclasses + 1)[1:-1]})


def candidates(edges):
    """(name, edges, kinds) schedules to time: the persistent launch on the warp and on the duo
    instance; the per-class launches on either; the per-class launches with the longest class
    (and the two longest) on the wide instance and the rest on the warp or the duo instance;
    and the longest class on the warp instance with the rest on the duo instance."""
    n = len(edges) + 1
    e = list(edges)
    out = [("persistent, warp instance", [], [0]), ("persistent, duo instance", [], [2]),
           ("per-class, warp instance", e, [0] * n), ("per-class, duo instance", e, [2] * n)]
    for w in range(1, min(2, n - 1) + 1):
        out.append((f"per-class, longest {w} on the wide instance, the rest warp", e, [1] * w + [0] * (n - w)))
        out.append((f"per-class, longest {w} on the wide instance, the rest duo", e, [1] * w + [2] * (n - w)))
    if n > 1:
        out.append(("per-class, longest on the warp instance, the rest duo", e, [0] + [2] * (n - 1)))
    return out


def time_schedule(ctx: Context, self_cmp: bool, edges, kinds, repeats=2):
    """Aligner device time (ms, both orientations) of the loaded blocks under one schedule."""
    ctx.set_align_schedule(edges, kinds)
    best = None
    for _ in range(repeats):
        ctx.reset_overlap_buffer()
        run_loaded(ctx, self_cmp)
        st = ctx.stats()
        ms = float(sum(st["ms_align"]))
        best = ms if best is None else min(best, ms)
    return best, int(st["records"])


def tune(ctx: Context, A, B=None, nclasses=3, repeats=2):
    """Times the candidate schedules on the loaded blocks (A in slot 0; B in slot 1, or None
    for A against itself), leaves the fastest set on ctx and returns a report: every
    candidate's aligner time and the choice."""
    self_cmp = B is None
    edges = length_edges(A, B, nclasses)
    report = []
    records = set()
    for name, e, k in candidates(edges):
        ms, nrec = time_schedule(ctx, self_cmp, e, k, repeats)
        records.add(nrec)
        report.append({"schedule": name, "edges": e, "kinds": k, "align_ms": round(ms, 3)})
    if len(records) != 1:
        raise RuntimeError(f"schedules gave different record counts: {sorted(records)}")
    best = min(report, key=lambda r: r["align_ms"])
    ctx.set_align_schedule(best["edges"], best["kinds"])
    ctx.reset_overlap_buffer()
    return {"chosen": best["schedule"], "edges": best["edges"], "kinds": best["kinds"], "candidates": report}


__all__ = ["length_edges", "candidates", "time_schedule", "tune"]

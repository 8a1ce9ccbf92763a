"""CPU restatement of LAsort (dalign/LAsort.c) -- TEST INFRASTRUCTURE ONLY.

Reads a .las file, orders its records by SORT_OVL of LAsort.c:65-90 (aread, bread, abpos;
the reference's qsort leaves ties in no fixed order, this restatement keeps them in file
order) and writes each record's bytes unchanged (LAsort.c:223-246: the 40-byte header,
pad included, then the trace), into the output path.
"""
from __future__ import annotations

import numpy as np


def read_records(path):
    with open(path, "rb") as f:
        data = f.read()
    n = int(np.frombuffer(data[:8], "<i8")[0])
    ts = int(np.frombuffer(data[8:12], "<i4")[0])
    tb = 1 if ts <= 125 else 2          # TRACE_XOVR (dalign/align.h)
    recs, o = [], 12
    for _ in range(n):
        h = np.frombuffer(data[o:o + 40], "<i4")
        ln = 40 + int(h[0]) * tb
        recs.append((int(h[7]), int(h[8]), int(h[2]), data[o:o + ln]))
        o += ln
    return n, ts, recs


def las_sort(src, dst):
    n, ts, recs = read_records(src)
    order = sorted(range(n), key=lambda i: recs[i][:3])   # Python's sort is stable
    with open(dst, "wb") as f:
        f.write(np.int64(n).tobytes())
        f.write(np.int32(ts).tobytes())
        for i in order:
            f.write(recs[i][3])
    return n


def las_merge(srcs, dst):
    """LAmerge's result (utils/LAmerge.c): the records of all inputs ordered by SORT_OVL of
    utils/LAmergeUtils.c:50-79 (aread, bread, orientation, abpos); LAmerge's heap leaves ties
    in no fixed order, this restatement keeps them in input order."""
    recs, ts = [], None
    for s in srcs:
        n, t, r = read_records(s)
        if ts is not None and t != ts:
            raise ValueError("trace spacings differ")
        ts = t
        recs += r
    def key(i):
        a, b, ab, raw = recs[i]
        comp = int(np.frombuffer(raw[24:28], "<u4")[0]) & 1
        return (a, b, comp, ab)
    order = sorted(range(len(recs)), key=key)
    with open(dst, "wb") as f:
        f.write(np.int64(len(recs)).tobytes())
        f.write(np.int32(ts).tobytes())
        for i in order:
            f.write(recs[i][3])
    return len(recs)

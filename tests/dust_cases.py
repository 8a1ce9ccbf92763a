"""The DBdust fixtures (tests/golden/dust): the runs and a reader for the track files."""
import json
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dust")


def runs():
    meta = json.load(open(os.path.join(GOLD, "dust.json")))
    out = []
    for r in meta["runs"]:
        kw = dict(window=64, thresh=2.0, mflag=10, biased=False)
        for f in r["flags"]:
            if f == "-b":
                kw["biased"] = True
            elif f.startswith("-w"):
                kw["window"] = int(f[2:])
            elif f.startswith("-t"):
                kw["thresh"] = float(f[2:])
            elif f.startswith("-m"):
                kw["mflag"] = int(f[2:])
        out.append((r["track"], r["db"], kw))
    return out


def read_track(base):
    """(nreads, anno int64[n+1], data int32) of `base`.anno / `base`.data."""
    a = open(base + ".anno", "rb").read()
    n, size = np.frombuffer(a[:8], "<i4")
    assert size == 8
    return int(n), np.frombuffer(a[8:], "<i8"), np.fromfile(base + ".data", "<i4")

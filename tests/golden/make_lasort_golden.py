"""Regenerates the LAsort fixtures from the reference LAsort (built from source by
oracle/Makefile into oracle/_ref):

* lasort/cat.las -- the three .las files of block 1 of hpc_3blocks, concatenated and with
  their records shuffled (seeded), 1-byte trace points;
* lasort/s200.las -- 400 shuffled records of self_s200_t20's .las (2-byte trace points);
* lasort/*.S.las -- what the reference LAsort writes for each.

Run from the repository root:  make -C oracle ref && python tests/golden/make_lasort_golden.py
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from marvel_b200 import dazzdb  # noqa: E402


def write_raw(path, tspace, raw_records):
    with open(path, "wb") as f:
        f.write(np.int64(len(raw_records)).tobytes())
        f.write(np.int32(tspace).tobytes())
        for r in raw_records:
            f.write(r)


def raw_records(path):
    """The byte string of each record of a .las file (40-byte header + trace), pad included."""
    with open(path, "rb") as f:
        data = f.read()
    n = int(np.frombuffer(data[:8], "<i8")[0])
    ts = int(np.frombuffer(data[8:12], "<i4")[0])
    tb = 1 if ts <= 125 else 2
    out, o = [], 12
    for _ in range(n):
        tlen = int(np.frombuffer(data[o:o + 4], "<i4")[0])
        out.append(data[o:o + 40 + tlen * tb])
        o += 40 + tlen * tb
    return ts, out


def main():
    d = os.path.join(HERE, "lasort")
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    rng = np.random.default_rng(11)
    recs, ts = [], None
    for n in ("G.1.G.1.las", "G.1.G.2.las", "G.1.G.3.las"):
        ts, r = raw_records(os.path.join(HERE, "hpc_3blocks", "001_00001", n))
        recs += r
    recs = [recs[i] for i in rng.permutation(len(recs))]
    write_raw(os.path.join(d, "cat.las"), ts, recs)
    ts, r = raw_records(os.path.join(HERE, "self_s200_t20", "001_00001", "G.1.G.1.las"))
    r = [r[i] for i in rng.permutation(len(r))[:400]]
    write_raw(os.path.join(d, "s200.las"), ts, r)
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "LAsort"), "cat.las", "s200.las"], cwd=d, check=True)
    for n in ("cat", "s200"):
        assert dazzdb.read_las(os.path.join(d, n + ".S.las"))[1].size > 0


if __name__ == "__main__":
    main()

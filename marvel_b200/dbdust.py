"""DBdust on the GPU: `python -m marvel_b200.dbdust [-b] [-w<int(64)>] [-t<double(2.)>] [-m<int(10)>] <path:db>`

Writes the `dust` interval track of a DB or of one block (`G.2`) -- `.G.dust.anno` /
`.G.dust.data`, or `.G.2.dust.anno` / `.G.2.dust.data` -- in the layout DBdust writes
(db/DBdust.c:182-213, 476-487): anno = int nreads, int 8, then nreads + 1 int64 byte
offsets into data; data = (begin, end) int32 pairs.  The scan runs on the device
(gd_dust).  Unlike DBdust, an existing track is always rewritten (DBdust resumes a track
that covers fewer reads than the DB).
"""
from __future__ import annotations

import getopt
import os
import sys

import numpy as np

from . import Context, dazzdb


def track_paths(db: str, name: str = "dust"):
    """(anno, data) paths for db (a DB or a block `root.n`), DBdust's naming."""
    d = os.path.dirname(db) or "."
    root = os.path.basename(db)
    if root.endswith(".db"):
        root = root[:-3]
    return os.path.join(d, f".{root}.{name}.anno"), os.path.join(d, f".{root}.{name}.data")


def write_track(anno_path, data_path, anno, data):
    n = anno.size - 1
    with open(anno_path, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.int32(8).tobytes())
        f.write(anno.astype("<i8").tobytes())
    with open(data_path, "wb") as f:
        f.write(data.astype("<i4").tobytes())


def dust_db(db: str, window=64, thresh=2.0, mflag=10, biased=False, ctx: Context | None = None):
    blk = dazzdb.open_block(db if not db.endswith(".db") else db[:-3])
    own = ctx is None
    ctx = ctx or Context()
    try:
        ctx.load_block(0, blk)
        anno, data = ctx.dust(0, blk.freq, window, thresh, mflag, biased)
    finally:
        if own:
            ctx.close()
    a, d = track_paths(db)
    write_track(a, d, anno, data)
    return anno, data


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    try:
        opts, args = getopt.getopt(argv, "bw:t:m:")
    except getopt.GetoptError as e:
        print(f"[ERROR] {e}", file=sys.stderr)
        return 1
    o = dict(window=64, thresh=2.0, mflag=10, biased=False)
    for k, v in opts:
        if k == "-b":
            o["biased"] = True
        elif k == "-w":
            o["window"] = int(v)
        elif k == "-t":
            o["thresh"] = float(v)
        elif k == "-m":
            o["mflag"] = int(float(v))
    if not args:
        print("usage: [-b] [-w <int(64)>] [-t<double(2.)>] [-m<int(10)>] <path:db|dam>", file=sys.stderr)
        return 1
    dust_db(args[0], **o)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

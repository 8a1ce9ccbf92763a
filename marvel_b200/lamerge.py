"""LAmerge on the GPU: `python -m marvel_b200.lamerge [-v] [-s] [-k] [-n <int>] <db> <merged.las> <dir | .las files>`

Merges sorted .las files (all `*.las` of a directory, names starting with `.` excluded, as
utils/LAmergeUtils.c:574-626 collects them, or the files given) into one file ordered by
(aread, bread, orientation, abpos) -- LAmerge's order (utils/LAmergeUtils.c:50-79).  The
merge is one device sort of all records (gd_las_merge), so -n (files per merge round),
-s (sort inputs first) and -k (keep intermediate files) have nothing to do and are
accepted for compatibility; a single input is copied, as LAmerge does.  Ties of the key,
which LAmerge's heap leaves in no fixed order, come out by (aepos, bbpos), then input order.
"""
from __future__ import annotations

import getopt
import os
import shutil
import sys

from . import Context


def inputs(args):
    files = []
    for a in args:
        if os.path.isdir(a):
            files += sorted(os.path.join(a, f) for f in os.listdir(a) if f.endswith(".las") and not f.startswith("."))
        else:
            files.append(a)
    return files


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    try:
        opts, args = getopt.getopt(argv, "vskn:")
    except getopt.GetoptError as e:
        print(f"[ERROR] - LAmerge: {e}", file=sys.stderr)
        return 1
    verbose = any(k == "-v" for k, _ in opts)
    if len(args) < 3:
        print("usage: lamerge [-v] [-s] [-k] [-n <int>] <db> <merged.las> <dir | .las files>", file=sys.stderr)
        return 1
    out = args[1]
    files = inputs(args[2:])
    if not files:
        print("[WARNING] - LAmerge: No input files. Nothing to do!", file=sys.stderr)
        return 0
    if len(files) == 1:
        shutil.copyfile(files[0], out)
        return 0
    ctx = Context()
    try:
        n = ctx.las_merge(files, out)
    finally:
        ctx.close()
    if verbose:
        print(f"merged {len(files)} files, {n:,} records -> {out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

"""LAsort on the GPU: `python -m marvel_b200.lasort [-v] <align:las> ...`

Each U.las is sorted by (aread, bread, abpos) into U.S.las next to it, as dalign/LAsort.c
does (:139-256); the sort runs on the device (gd_las_sort).  Records keep their bytes; ties
of the reference's sort key, which its qsort leaves in no fixed order, come out ordered by
(aepos, bbpos) and then by their order in the input file.
"""
from __future__ import annotations

import os
import sys

from . import Context


def out_name(path: str) -> tuple[str, str]:
    """(input, output) paths as LAsort builds them: PathTo(arg) / Root(arg, ".las") + .las/.S.las."""
    d = os.path.dirname(path) or "."
    root = os.path.basename(path)
    if root.endswith(".las"):
        root = root[:-4]
    return os.path.join(d, root + ".las"), os.path.join(d, root + ".S.las")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    verbose = "-v" in argv
    files = [a for a in argv if not a.startswith("-")]
    if not files:
        print("Usage: lasort [-v] <align:las> ...", file=sys.stderr)
        return 1
    ctx = Context()
    try:
        for a in files:
            src, dst = out_name(a)
            n = ctx.las_sort(src, dst)
            if verbose:
                print(f"  {os.path.basename(src)[:-4]}: {n:,} records")
    finally:
        ctx.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

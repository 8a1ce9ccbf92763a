"""Compute_Trace_PTS fixtures from the reference itself.

For every .las file of the daligner golden cases, oracle/_ref/trace_pts_harness (built by
oracle/Makefile from oracle/trace_pts_harness.c and the reference's dalign/align.c) runs the
reference's Compute_Trace_PTS (dalign/align.c:5286-5397) on each record, as LAcheck -a does,
and prints the diffs it computes.  They are stored per file in trace_pts.npz (key
"<case>/<las path>", int32 per record in file order).  Run from the repository root:

    make -C oracle ref && python tests/golden/make_trace_pts_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from golden_cases import cases, load  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "trace_pts_harness")


def main():
    out = {}
    for name in cases():
        d, meta = load(name)
        for las in meta["las"]:
            p = subprocess.run([HARNESS, "G", las], cwd=d, check=True, capture_output=True, text=True)
            diffs = np.array([int(x) for x in p.stdout.split()], np.int32)
            out[f"{name}/{las}"] = diffs
            print(name, las, diffs.size, int(diffs.sum()))
    np.savez_compressed(os.path.join(HERE, "trace_pts.npz"), **out)


if __name__ == "__main__":
    main()

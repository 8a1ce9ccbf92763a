"""Records the reference daligner's -v report (stdout) for some golden cases.

For each case the DB is copied to a scratch directory, the reference (built from source by
oracle/Makefile into oracle/_ref) runs with -v and the case's flags, and its stdout is
written to <case>/verbose.txt.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_verbose_golden.py
"""
from __future__ import annotations

import glob
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "daligner")

CASES = ["self_s200_t20", "pair_blocks", "self_asym_lowmem", "pair_dust_biased"]


def make(name):
    d = os.path.join(HERE, name)
    with open(os.path.join(d, "case.json")) as f:
        meta = json.load(f)
    with tempfile.TemporaryDirectory() as t:
        for f in glob.glob(os.path.join(d, "*")) + glob.glob(os.path.join(d, ".*")):
            if os.path.isfile(f):
                shutil.copy(f, t)
        r = subprocess.run([REF, "-v", "-j4"] + meta["flags"] + meta["blocks"], cwd=t, check=True,
                           capture_output=True, text=True)
    with open(os.path.join(d, "verbose.txt"), "w") as f:
        f.write(r.stdout)
    return len(r.stdout)


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        print(n, make(n))

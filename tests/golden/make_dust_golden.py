"""Regenerates the DBdust fixtures from the reference DBdust (built from source by
oracle/Makefile into oracle/_ref): one small DB with tandem repeats, split in two blocks,
and the interval tracks DBdust writes for it --

  dust   the whole DB, default options            dustb  the whole DB, -b (biased)
  dustw  the whole DB, -w32 -t1.5 -m8              (block) .G.2.dust.*: block 2, default

each renamed after the run (DBdust always writes a track called `dust`).  Run from the
repository root:  make -C oracle ref && python tests/golden/make_dust_golden.py
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from marvel_b200 import dazzdb, synth  # noqa: E402

DUST = os.path.join(ROOT, "oracle", "_ref", "DBdust")
# DBdust resumes an existing `dust` track instead of rewriting it, so the renamed variants
# run first, each on a DB without a `dust` track
RUNS = [("dustb", "G", ["-b"]), ("dustw", "G", ["-w32", "-t1.5", "-m8"]), ("dust", "G", []), ("dust", "G.2", [])]


def main():
    d = os.path.join(HERE, "dust")
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    reads, _ = synth.generate("tiny_tandem", 0.6)
    dazzdb.write_db(os.path.join(d, "G"), reads, 0.3)
    for name, db, flags in RUNS:
        subprocess.run([DUST] + flags + [db], cwd=d, check=True, stdout=subprocess.DEVNULL)
        if name != "dust":
            for ext in ("anno", "data"):
                os.rename(os.path.join(d, f".{db}.dust.{ext}"), os.path.join(d, f".{db}.{name}.{ext}"))
    with open(os.path.join(d, "dust.json"), "w") as f:
        json.dump({"workload": "tiny_tandem", "scale": 0.6, "block_mbp": 0.3,
                   "runs": [{"track": n, "db": db, "flags": fl} for n, db, fl in RUNS]}, f, indent=1)


if __name__ == "__main__":
    main()

"""Regenerates the HPCdaligner fixtures from the reference, built from source by
oracle/Makefile into oracle/_ref:

* hpc_plans.json -- HPCdaligner's printed plan for a 4-block DB under several option sets;
* hpc_3blocks/ -- a 3-block DB, every .las file its default plan's daligner calls write
  (run with the reference daligner), and the merged G.n.las files the plan's LAmerge calls
  write (reference LAmerge), for the multi-block driver's and LAmerge's tests.

Run from the repository root:  make -C oracle ref && python tests/golden/make_hpc_golden.py
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from marvel_b200 import dazzdb, synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")

PLAN_ARGS = [
    "G", "-X --dal 2 G", "--dal 2 --dalDiag 1 -k16 -A G 2-4", "-v -I -e0.8 -l500 -s50 -M8 -T G",
    "-X -A -T -M8 G 1-3", "-mdust -mtan -t20 -h40 -w5 --dal 3 --mrg 4 -S -K G", "-vv --dal 1 G 2",
    "-X --dal 3 G 2-4", "-r3 -j8 --dalDiag 2 --dal 1 G", "sub/G 2-3",
]


def plans():
    with tempfile.TemporaryDirectory() as d:
        reads, _ = synth.generate("tiny")
        os.makedirs(os.path.join(d, "sub"))
        dazzdb.write_db(os.path.join(d, "G"), reads, 0.2)
        dazzdb.write_db(os.path.join(d, "sub", "G"), reads, 0.2)
        out = []
        for a in PLAN_ARGS:
            r = subprocess.run([os.path.join(REF, "HPCdaligner")] + a.split(), cwd=d, check=True,
                               capture_output=True, text=True)
            out.append({"args": a, "plan": r.stdout})
    with open(os.path.join(HERE, "hpc_plans.json"), "w") as f:
        json.dump({"blocks": 4, "plans": out}, f, indent=1)


def three_blocks():
    d = os.path.join(HERE, "hpc_3blocks")
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    reads, _ = synth.generate("tiny", 0.8)
    dazzdb.write_db(os.path.join(d, "G"), reads, 0.2)
    plan = subprocess.run([os.path.join(REF, "HPCdaligner"), "G"], cwd=d, check=True, capture_output=True,
                          text=True).stdout
    calls = [ln.split()[1:] for ln in plan.splitlines() if ln.startswith("daligner ")]
    for c in calls:
        subprocess.run([os.path.join(REF, "daligner")] + c, cwd=d, check=True, stdout=subprocess.DEVNULL)
    las = sorted(os.path.relpath(os.path.join(r, f), d) for r, _, fs in os.walk(d) for f in fs if f.endswith(".las"))
    # the plan's LAmerge calls: one merged file per block from its directory
    merges = [ln.split()[1:] for ln in plan.splitlines() if ln.startswith("LAmerge ")]
    for m in merges:
        subprocess.run([os.path.join(REF, "LAmerge")] + m, cwd=d, check=True, stdout=subprocess.DEVNULL)
    with open(os.path.join(d, "hpc.json"), "w") as f:
        json.dump({"workload": "tiny", "scale": 0.8, "block_mbp": 0.2, "plan": plan, "las": las,
                   "merged": [m[-2] for m in merges], "merge_dirs": [m[-1] for m in merges]}, f, indent=1)


if __name__ == "__main__":
    plans()
    three_blocks()

"""Digests of the reference daligner's output on the full-size synthetic workloads.

The workloads (marvel_b200.synth: seeded genomes and reads, written as DBs) are too large
to commit, so what is committed is, per workload, what the reference daligner (built from
source by oracle/Makefile into oracle/_ref) writes for its comparison (block 1 against
itself, or block 1 against block 2 with the reference DBdust's track): the record count,
the trace spacing and dazzdb.las_digest of its .las files together -- a
SHA-256 over the records (every field but the uninitialised pad word, and every trace
byte) in a canonical order, so that any order among tied sort keys gives the same
digest.  With --cells the reference built with its own wave counters
(oracle/_ref/daligner_wavestats, -j1 so that the counts are exact) also gives the
aligner's cell and wave counts.

The GPU test (tests/test_gpu_config_parity.py) regenerates the same DBs from the same
seeds and compares its own output's digest with these.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_config_digests.py [--cells] [names...]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from marvel_b200 import dazzdb, synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(HERE, "config_digests.json")
FLAGS = ["-M32", "-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"]

# name: (workload, genome scale, mask tracks, what it is).  A workload split into blocks is
# compared block 1 against block 2 when it has two blocks generated (cfg5), else block 1
# against itself.
CONFIGS = {
    "cfg1": ("cfg1", 1.0, [], "1 Mbp genome, 20x, mean 8 kbp: the CPU-runnable block"),
    "cfg2": ("cfg2", 1.0, [], "4.6 Mbp + repeats, 25x, mean 10 kbp: the benchmarked block"),
    "cfg3": ("cfg3", 1.0, [], "10 Mbp genome, 30x, 1-150 kbp reads with homopolymer-biased deletions"),
    "cfg4_x0.25": ("cfg4", 0.25, [], "cfg4's model on a 5 Mbp genome (10% interspersed 1-8 kbp repeats at "
                                    "5-15%), block 1 of 50 Mbp vs itself"),
    "cfg5_x0.02": ("cfg5", 0.02, ["dust"], "cfg5's model on a 4 Mbp diploid genome (35% interspersed, 2% tandem "
                                          "repeats), block 1 vs block 2 of 8 Mbp, -mdust"),
}


def threads():
    n = os.cpu_count() or 1
    j = 1
    while j * 2 <= n:
        j *= 2
    return j


def las_set_digest(paths):
    """dazzdb.las_digest over the records of several .las files together."""
    import numpy as np
    recs, tbs, toffs, base, tspace = [], [], [], 0, None
    for p in paths:
        tspace, r, tb, toff = dazzdb.read_las_arrays(p)
        recs.append(r)
        tbs.append(tb)
        toffs.append(toff + base)
        base += tb.size
    d, n = dazzdb.las_digest(np.concatenate(recs), np.concatenate(tbs), np.concatenate(toffs),
                             1 if tspace <= 125 else 2)
    return tspace, d, n


def run(name, cells, cache):
    wl, scale, masks, desc = CONFIGS[name]
    blk = synth.cached_db(wl, 0, scale, cache)
    A = dazzdb.open_block(blk)
    pair = synth.WORKLOADS[wl].nblocks >= 2
    B = dazzdb.open_block(blk[:-2] + ".2") if pair else A
    src = os.path.dirname(blk)
    flags = [f"-m{m}" for m in masks] + FLAGS
    blocks = ["W.1", "W.2"] if pair else ["W.1", "W.1"]
    las = ["001_00001/W.1.W.2.las", "001_00002/W.2.W.1.las"] if pair else ["001_00001/W.1.W.1.las"]
    with tempfile.TemporaryDirectory() as d:
        for f in os.listdir(src):
            if (f.startswith("W.") or f.startswith(".W.")) and ".dust." not in f:
                os.symlink(os.path.join(src, f), os.path.join(d, f))
        for m in masks:   # the reference's own DBdust writes the track
            assert m == "dust"
            subprocess.run([os.path.join(REF, "DBdust"), "W"], cwd=d, check=True, stdout=subprocess.DEVNULL)
        t = time.perf_counter()
        subprocess.run([os.path.join(REF, "daligner"), f"-j{threads()}"] + flags + blocks, cwd=d, check=True,
                       stdout=subprocess.DEVNULL)
        wall = time.perf_counter() - t
        tspace, digest, n = las_set_digest([os.path.join(d, x) for x in las])
        rec = {"workload": wl, "scale": scale, "seed_offset": 0, "what": desc, "flags": " ".join(flags),
               "blocks": blocks, "masks": masks, "reads": int(A.nreads), "bases": int(A.totlen),
               "b_reads": int(B.nreads), "b_bases": int(B.totlen), "novl": n, "tspace": tspace, "sha256": digest,
               "reference_wall_s": round(wall, 1), "reference_threads": threads()}
        if cells:
            for x in las:
                shutil.rmtree(os.path.join(d, os.path.dirname(x)), ignore_errors=True)
            p = subprocess.run([os.path.join(REF, "daligner_wavestats"), "-j1"] + flags + blocks, cwd=d,
                               check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)
            m = re.search(r"WAVE_STATS cells (\d+) waves (\d+) widest (\d+)", p.stderr)
            rec.update(cells=int(m.group(1)), waves=int(m.group(2)), widest=int(m.group(3)))
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*", default=list(CONFIGS))
    ap.add_argument("--cells", action="store_true", help="also count cells with the WAVE_STATS build (-j1)")
    ap.add_argument("--cache", default=os.path.join(tempfile.gettempdir(), "marvel_b200_bench"))
    a = ap.parse_args()
    have = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            have = json.load(f)
    for name in a.names:
        rec = run(name, a.cells, a.cache)
        if not a.cells and name in have:
            for k in ("cells", "waves", "widest"):
                if k in have[name]:
                    rec[k] = have[name][k]
        have[name] = rec
        print(name, rec, flush=True)
        with open(OUT, "w") as f:
            json.dump(have, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main()

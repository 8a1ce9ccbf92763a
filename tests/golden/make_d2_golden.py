"""Regenerates the daligner2 (modimizer seeds) golden fixtures from the reference daligner2.

Each case is a small seeded synthetic DB (marvel_b200.dazzdb, byte-compatible with FA2db +
DBsplit) and the .las file(s) the reference daligner2, built from source by oracle/Makefile
into oracle/_ref, writes for it (under -P, in per-block folders <P>_<block>/).  Run from the
repository root:

    make -C oracle ref && python tests/golden/make_d2_golden.py
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

REF = os.path.join(ROOT, "oracle", "_ref", "daligner2")
DUST = os.path.join(ROOT, "oracle", "_ref", "DBdust")

BASE = ["-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"]
# name: (workload, genome scale, block size in Mbp, daligner2 flags, block arguments)
CASES = {
    "d2_self": ("tiny", 1.0, 200, BASE, ["G.1", "G.1"]),
    "d2_pair": ("tiny", 1.0, 0.35, BASE, ["G.1", "G.2"]),
    "d2_self_k16_w5": ("tiny", 0.7, 200, ["-k16", "-w5", "-h40", "-e.70", "-l1000", "-s100"], ["G.1", "G.1"]),
    "d2_self_k12_identity": ("tiny", 0.5, 200, ["-I", "-k12", "-w6", "-h30", "-e.70", "-l500", "-s100"],
                             ["G.1", "G.1"]),
    "d2_self_asym_t20": ("tiny", 0.7, 200, ["-A", "-t20"] + BASE, ["G.1", "G.1"]),
    "d2_self_hgap": ("tiny", 0.7, 200, ["-H6000"] + BASE, ["G.1", "G.1"]),
    "d2_self_s200_lowmem": ("tiny", 0.7, 200, ["-M0", "-k14", "-w6", "-h35", "-e.75", "-l800", "-s200"],
                            ["G.1", "G.1"]),
    "d2_pair_dust": ("tiny_tandem", 1.0, 0.4, ["-mdust"] + BASE, ["G.1", "G.2"]),
}


def make_case(name):
    wl, scale, bsize, flags, blocks = CASES[name]
    d = os.path.join(HERE, name)
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    reads, _ = synth.generate(wl, scale)
    dazzdb.write_db(os.path.join(d, "G"), reads, bsize)
    if any(f.startswith("-m") for f in flags):
        subprocess.run([DUST, "G"], cwd=d, check=True, stdout=subprocess.DEVNULL)
    mem = [] if any(f.startswith("-M") for f in flags) else ["-M32"]
    cmd = [REF, "-T4", "-Pout"] + mem + flags + blocks
    subprocess.run(cmd, cwd=d, check=True, stdout=subprocess.DEVNULL)
    las = []
    for root, _, files in os.walk(d):
        for f in files:
            if f.endswith(".las"):
                las.append(os.path.relpath(os.path.join(root, f), d))
    meta = {"workload": wl, "scale": scale, "block_mbp": bsize, "flags": mem + flags, "blocks": blocks,
            "las": sorted(las), "command": " ".join(["daligner2", "-T4", "-Pout"] + mem + flags + blocks)}
    with open(os.path.join(d, "case.json"), "w") as f:
        json.dump(meta, f, indent=1)
    return meta


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        print(n, make_case(n))

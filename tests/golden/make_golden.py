"""Regenerates the golden fixtures from the reference daligner.

Each case is a small seeded synthetic DB (written by marvel_b200.dazzdb, byte-compatible
with FA2db + DBsplit) and the .las file(s) the reference daligner, built from source by
oracle/Makefile into oracle/_ref, writes for it.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py
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

REF = os.path.join(ROOT, "oracle", "_ref", "daligner")

# name: (workload, genome scale, block size in Mbp, daligner flags, block arguments)
CASES = {
    "self_default": ("tiny", 1.0, 200, ["-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"], ["G.1", "G.1"]),
    "pair_blocks": ("tiny", 1.0, 0.35, ["-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"], ["G.1", "G.2"]),
    "self_s200_t20": ("tiny", 0.7, 200, ["-k14", "-w6", "-h35", "-e.75", "-l800", "-s200", "-t20"], ["G.1", "G.1"]),
    "self_k16_w5": ("tiny", 0.7, 200, ["-k16", "-w5", "-h40", "-e.70", "-l1000", "-s100"], ["G.1", "G.1"]),
    "self_identity": ("tiny", 0.5, 200, ["-I", "-k12", "-w6", "-h30", "-e.70", "-l500", "-s100"], ["G.1", "G.1"]),
    "self_asym_lowmem": ("tiny", 0.7, 200, ["-A", "-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100", "-M0"],
                         ["G.1", "G.1"]),
    # reads of 30-150 kbp: the seed scan's 50,000-bp panels (dalign/filter.c:1717-1745)
    "self_long_panels": ("long", 1.0, 200, ["-k14", "-w6", "-h35", "-e.75", "-l1000", "-s100"], ["G.1", "G.1"]),
    # tandem repeats masked by the reference DBdust track (-mdust), blocks of ~0.4 Mbp
    "pair_dust": ("tiny_tandem", 1.0, 0.4, ["-mdust", "-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"],
                  ["G.1", "G.2"]),
    # -b: frequency-weighted tuples on an AT-rich genome, whole reads and (with a dust track)
    # unmasked segments
    "self_biased": ("tiny_at", 1.0, 200, ["-b", "-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"], ["G.1", "G.1"]),
    "pair_dust_biased": ("tiny_at_tandem", 1.0, 0.4, ["-b", "-mdust", "-k14", "-w6", "-h35", "-e.70", "-l1000",
                                                      "-s100"], ["G.1", "G.2"]),
    "self_dust_biased_k12": ("tiny_skew_tandem", 1.0, 200, ["-b", "-mdust", "-k12", "-w6", "-h30", "-e.70", "-l800",
                                                            "-s100"], ["G.1", "G.1"]),
}
DUST = os.path.join(ROOT, "oracle", "_ref", "DBdust")


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
    cmd = [REF, "-j4", "-M32"] + flags + blocks
    subprocess.run(cmd, cwd=d, check=True, stdout=subprocess.DEVNULL)
    las = []
    for root, _, files in os.walk(d):
        for f in files:
            if f.endswith(".las"):
                las.append(os.path.relpath(os.path.join(root, f), d))
    meta = {"workload": wl, "scale": scale, "block_mbp": bsize, "flags": ["-M32"] + flags, "blocks": blocks,
            "las": sorted(las), "command": " ".join(["daligner", "-j4", "-M32"] + flags + blocks)}
    with open(os.path.join(d, "case.json"), "w") as f:
        json.dump(meta, f, indent=1)
    return meta


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        print(n, make_case(n))

"""The blocks of a synthetic workload's comparison, ready for the device path.

A workload (marvel_b200.synth) with two blocks generated is compared block 1 against block
2, any other one block 1 against itself; its mask tracks (synth.Workload.masks, e.g. the
dust track) are made once for the whole DB by this package's device DBdust
(marvel_b200.dbdust, byte-identical to the reference DBdust's files) and loaded into both
blocks, as daligner's -m does (dalign/daligner.c:385-442).
"""
from __future__ import annotations

import os

from . import dazzdb, synth


def track_exists(root: str, name: str) -> bool:
    d, b = os.path.split(root)
    return os.path.exists(os.path.join(d, f".{b}.{name}.anno"))


def blocks(workload: str, seed_offset: int = 0, scale: float = 1.0, cache: str | None = None):
    """(A, B) of the workload's comparison; B is None for a block against itself."""
    path = synth.cached_db(workload, seed_offset, scale, cache)
    w = synth.WORKLOADS[workload]
    root = path.rsplit(".", 1)[0]
    for m in w.masks:
        if m != "dust":
            raise ValueError(f"no generator for track {m}")
        if not track_exists(root, m):
            from . import dbdust
            dbdust.dust_db(root)
    A = dazzdb.open_block(path)
    B = dazzdb.open_block(path[:-2] + ".2") if w.nblocks >= 2 else None
    for m in w.masks:
        for blk in (A, B):
            if blk is not None:
                dazzdb.load_track(blk, m)
    return A, B

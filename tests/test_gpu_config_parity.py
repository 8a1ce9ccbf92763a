"""GPU parity at full workload size: the device path's output on the whole benchmarked
blocks equals the reference daligner's.

The blocks are regenerated from their seeds (marvel_b200.synth, the same DBs the benchmark
uses); tests/golden/config_digests.json holds, per block, what the reference daligner wrote
for it (record count, trace spacing and the order-free SHA-256 of its .las records, from
tests/golden/make_config_digests.py) and the reference's own wave-cell count (its
WAVE_STATS counters, -j1).  Bit-exact: every field of every record but the pad word, and
every trace byte; the cell count exactly.  Both on the default aligner schedule and with every
pair group on the duo instance."""
import json
import os

import numpy as np
import pytest

from marvel_b200 import dazzdb, synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "config_digests.json")) as _f:
    DIGESTS = json.load(_f)


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


def _sorted_like_write_overlap_buffer(recs):
    """SORT_OVL order (dalign/align.c:5786-5813): aread, bread, COMP, abpos non-decreasing."""
    k = np.stack([recs["aread"].astype(np.int64), recs["bread"].astype(np.int64),
                  (recs["flags"] & 1).astype(np.int64), recs["abpos"].astype(np.int64)], 1)
    d = np.diff(k, axis=0)
    first = np.argmax(d != 0, axis=1)
    lead = d[np.arange(d.shape[0]), first]
    return bool((lead >= 0).all())


@pytest.mark.parametrize("kinds", [None, [2]], ids=["warp", "duo"])
@pytest.mark.parametrize("name", sorted(DIGESTS))
def test_full_block_equals_reference(mb, name, kinds):
    want = DIGESTS[name]
    path = synth.cached_db(want["workload"], want["seed_offset"], want["scale"])
    A = dazzdb.open_block(path)
    pair = want.get("blocks", ["W.1", "W.1"])[1] != "W.1"
    B = dazzdb.open_block(path[:-2] + ".2") if pair else None
    assert (A.nreads, int(A.totlen)) == (want["reads"], want["bases"]), "the generator gave another block"
    for m in want.get("masks", []):
        # the track made by this package's device DBdust (byte-identical to the reference's)
        from marvel_b200 import dbdust
        assert m == "dust"
        dbdust.dust_db(path.rsplit(".", 1)[0])
        for blk in (A, B):
            if blk is not None:
                dazzdb.load_track(blk, m)
    ctx = mb.Context()
    if kinds is not None:
        ctx.set_align_schedule([], kinds)
    recs, tr = mb.daligner_block(ctx, A, B, k=14, w=6, h=35, e=0.70, l=1000, s=100, M=32)
    st = ctx.stats()
    ctx.close()
    assert want["tspace"] == 100
    digest, n = dazzdb.las_digest(recs, tr, recs["toff"], 1)
    assert n == want["novl"], f"{name}: {n} records, the reference wrote {want['novl']}"
    assert digest == want["sha256"], f"{name}: same count, different records"
    if not pair:   # a pair's buffer holds both files' records, each file sorted on its own
        assert _sorted_like_write_overlap_buffer(recs)
    if "cells" in want:
        assert int(sum(st["cells"])) == want["cells"], f"{name}: wave cells differ from the reference's WAVE_STATS"

"""DB and .las formats (CPU)."""
import os

import numpy as np

from golden_cases import GOLDEN, cases, load
from marvel_b200 import dazzdb, synth


def test_db_writer_reproduces_golden_db(tmp_path):
    # the committed DBs were written by the same seeded generator: regenerating must give the same bytes
    d, meta = load("pair_blocks")
    reads, _ = synth.generate(meta["workload"], meta["scale"])
    dazzdb.write_db(str(tmp_path / "G"), reads, meta["block_mbp"])
    for f in (".G.bps", "G.db"):
        assert open(tmp_path / f, "rb").read() == open(os.path.join(d, f), "rb").read(), f
    a = open(tmp_path / ".G.idx", "rb").read()
    b = open(os.path.join(d, ".G.idx"), "rb").read()
    assert a[:32] == b[:32]
    ra = np.frombuffer(a[88:], dazzdb.HITS_READ_DTYPE)
    rb = np.frombuffer(b[88:], dazzdb.HITS_READ_DTYPE)
    assert (ra["rlen"] == rb["rlen"]).all() and (ra["boff"] == rb["boff"]).all()


def test_block_loading_layout():
    d, meta = load("pair_blocks")
    b1 = dazzdb.open_block(os.path.join(d, "G.1"))
    b2 = dazzdb.open_block(os.path.join(d, "G.2"))
    assert b1.ufirst == 0 and b2.ufirst == b1.nreads and b1.part == 1 and b2.part == 2
    for b in (b1, b2):
        assert b.bases[0] == 4
        for i in range(b.nreads):
            o = int(b.boff[i]) + 1
            assert b.bases[o - 1] == 4 and b.bases[o + b.rlen[i]] == 4
            assert b.bases[o:o + b.rlen[i]].max() <= 3
        assert b.maxlen == b.rlen.max() and b.totlen == b.rlen.sum()


def test_complement_is_an_involution():
    d, _ = load("self_default")
    b = dazzdb.open_block(os.path.join(d, "G.1"))
    b.mask = [[(5, 40), (100, 120)]] * b.nreads
    c = dazzdb.complement_block(b)
    cc = dazzdb.complement_block(c)
    assert (cc.bases == b.bases).all() and cc.mask == b.mask
    r0 = b.read(0)
    assert (c.read(0) == 3 - r0[::-1]).all()


def test_golden_las_files_are_well_formed():
    for name in cases():
        d, meta = load(name)
        for las in meta["las"]:
            ts, recs, traces = dazzdb.read_las(os.path.join(d, las))
            tb_pairs = [t.size // 2 for t in traces]
            for r, t in zip(recs, traces):
                assert r["tlen"] == t.size and r["tlen"] % 2 == 0
                # Check_Trace_Points (dalign/align.c:3419-3449): b deltas sum to the b span
                if ts <= 125 and t.size:
                    assert int(t[1::2].sum()) == int(r["bepos"] - r["bbpos"])
            assert len(tb_pairs) == recs.size

"""GPU parity of daligner -b, the frequency-weighted tuples of biased_tuple_thread
(dalign/filter.c:492-633): the index, its complement and the hits against the oracle, bit for
bit, over whole reads and over a mask track's segments, for 32- and 64-bit codes, with -t, and
with values too wide to pack (read, position) in 32 bits.  The .las goldens of -b runs of the
reference are covered by the golden tests."""
import os

import numpy as np
import pytest

from golden_cases import load
from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


def _ctx(mb, A, k=14, t=0):
    ctx = mb.Context()
    ctx.set_biased(True)
    ctx.set_filter_params(k, 6, t, 35)
    ctx.new_align_spec(0.70, 100, A.freq)
    ctx.set_globals(2000, False, 32 << 30)
    return ctx


def _same_index(ctx, slot, blk, p):
    import oracle
    n = ctx.sort_kmers(slot)
    gc, gr, gp = ctx.get_kmers(slot, n)
    oc, orr, op = oracle.sort_kmers(blk, p)
    assert n == oc.size
    assert (gc == oc).all() and (gr == orr).all() and (gp == op).all()
    return n


@pytest.mark.parametrize("name,k,t,track", [
    ("self_biased", 14, 0, None),
    ("self_biased", 20, 0, None),
    ("self_biased", 12, 8, None),
    ("self_dust_biased_k12", 12, 0, "dust"),
    ("self_dust_biased_k12", 16, 0, "dust"),
])
def test_biased_index_and_hits_match_oracle(mb, name, k, t, track):
    import oracle
    d, _ = load(name)
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    if track:
        dazzdb.load_track(A, track)
    p = oracle.make_params(A.freq, k=k, t=t, biased=True)
    ctx = _ctx(mb, A, k, t)
    ctx.load_block(0, A)
    n = _same_index(ctx, 0, A, p)
    assert n > 0
    ctx.match_filter(0, 0, 1)
    gh = ctx.get_hits()
    oh, limit = oracle.match_hits(A, A, p, True)
    assert gh.shape == oh.shape and (gh == oh).all()
    # the complement's tuples are weighted with the same (A block) table
    ctx.complement_block(0, 2)
    _same_index(ctx, 2, dazzdb.complement_block(A), p)
    ctx.close()


def test_biased_tuples_at_segment_ends(mb):
    """Random mask intervals, adjacent and empty ones included: the tracked scan keeps a
    window that growing pushed onto a segment's end at that end (dalign/filter.c:545-551)."""
    import oracle
    d, _ = load("self_biased")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    rng = np.random.default_rng(5)
    mask = []
    for i in range(A.nreads):
        L = int(A.rlen[i])
        cuts = np.sort(rng.choice(L, size=2 * int(rng.integers(0, 12)), replace=False)).tolist()
        iv = [(cuts[j], cuts[j + 1]) for j in range(0, len(cuts), 2)]
        if i % 5 == 0 and iv:
            b, e = iv[-1]
            iv.append((e, e))                       # empty
            if e + 40 < L:
                iv.append((e, e + 40))              # adjacent to the previous one
        mask.append(iv)
    A.mask = mask
    p = oracle.make_params(A.freq, biased=True)
    ctx = _ctx(mb, A)
    ctx.load_block(0, A)
    n = ctx.sort_kmers(0)
    _, gr, gp = ctx.get_kmers(0, n)
    ends = {(r, b) for r, iv in enumerate(mask) for (b, e) in iv} | {(r, int(A.rlen[r])) for r in range(A.nreads)}
    assert sum((int(r), int(q)) in ends for r, q in zip(gr, gp)) > 0
    _same_index(ctx, 0, A, p)
    ctx.close()


def _block(reads, freq):
    rlen = np.array([r.size for r in reads], np.int32)
    boff = np.zeros(len(reads) + 1, np.int64)
    boff[1:] = np.cumsum(rlen.astype(np.int64) + 1)
    bases = np.full(int(boff[-1]) + 1, 4, np.uint8)
    for i, r in enumerate(reads):
        bases[boff[i] + 1:boff[i] + 1 + r.size] = r
    return dazzdb.Block(bases=bases, boff=boff, rlen=rlen, ufirst=0, part=1, freq=np.asarray(freq, np.float32),
                        maxlen=int(rlen.max()), totlen=int(rlen.sum()))


def test_biased_index_with_unpacked_values(mb):
    """2^17 + 1 reads and a 40 kbp read: read and position need 34 bits, so the sort carries
    entry indices and the index is gathered from the scan's (read, position) arrays."""
    import oracle
    rng = np.random.default_rng(9)
    probs = np.array([0.35, 0.15, 0.15, 0.35])
    reads = [rng.choice(4, size=int(rng.integers(14, 30)), p=probs).astype(np.uint8) for _ in range((1 << 17) + 1)]
    reads.append(rng.choice(4, size=40000, p=probs).astype(np.uint8))
    A = _block(reads, [0.35, 0.15, 0.15, 0.35])
    p = oracle.make_params(A.freq, biased=True)
    ctx = _ctx(mb, A)
    ctx.load_block(0, A)
    assert _same_index(ctx, 0, A, p) > 0
    ctx.close()


def test_biased_flag_rules(mb):
    d, _ = load("self_biased")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.set_variant(2, 0)
    with pytest.raises(RuntimeError):
        ctx.set_biased(True)
    ctx.set_variant(1, 0)
    ctx.set_biased(True)
    with pytest.raises(RuntimeError):
        ctx.set_variant(2, 0)
    ctx.set_filter_params(14, 6, 0, 35)
    ctx.new_align_spec(0.70, 100, [0.5, 0.5, 0.0, 0.0])
    ctx.load_block(0, A)
    with pytest.raises(RuntimeError, match=r"\(0, 1\]"):
        ctx.sort_kmers(0)
    ctx.close()

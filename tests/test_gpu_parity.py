"""GPU parity: the sm_100a path against the reference's golden .las files and the oracle.

Bit-exact for everything (integer work): .las records and every trace byte, the k-mer
index, the sorted hit list, and single Local_Alignment calls."""
import os

import numpy as np
import pytest

import daligner_run
from golden_cases import cases, load
from marvel_b200 import dazzdb, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


@pytest.mark.parametrize("name", cases())
def test_gpu_matches_reference_golden(mb, name, tmp_path):
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu")
    assert sorted(names) == sorted(meta["las"])
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


def _ctx(mb, A, k=14, w=6, t=0, h=35):
    ctx = mb.Context()
    ctx.set_filter_params(k, w, t, h)
    ctx.new_align_spec(0.70, 100, A.freq)
    ctx.set_globals(2000, False, 32 << 30)
    return ctx


@pytest.mark.parametrize("name", ["self_default", "pair_blocks", "self_long_panels"])
def test_wide_band_kernel_matches_reference_golden(mb, name, tmp_path):
    """The golden cases with a 32-diagonal main kernel, so that many pair groups go to the
    wide kernel: the .las files are still the reference's."""
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu", wave_limit=32)
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.parametrize("name,k", [("self_default", 14), ("self_k16_w5", 16)])
def test_kmer_index_and_hits_match_oracle(mb, name, k):
    import oracle
    d, _ = load(name)
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    p = oracle.make_params(A.freq, k=k)
    ctx = _ctx(mb, A, k=k)
    ctx.load_block(0, A)
    n = ctx.sort_kmers(0)
    gc, gr, gp = ctx.get_kmers(0, n)
    oc, orr, op = oracle.sort_kmers(A, p)
    assert n == oc.size
    assert (gc == oc).all() and (gr == orr).all() and (gp == op).all()
    ctx.match_filter(0, 0, 1)
    gh = ctx.get_hits()
    oh, limit = oracle.match_hits(A, A, p, True)
    assert gh.shape == oh.shape and (gh == oh).all()
    assert ctx.stats()["limit"][0] == limit
    ctx.close()


@pytest.mark.parametrize("k", [12, 16])
def test_masked_index_keeps_poly_t(mb, k):
    """k a multiple of 4 with a mask track: the masked slots' all-ones key must not take the
    place of real poly-T k-mers (the oracle lists the unmasked k-mers only)."""
    import oracle
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    A.bases = A.bases.copy()
    mask = []
    for i in range(A.nreads):
        o = int(A.boff[i]) + 1
        if i % 3 == 0:
            A.bases[o + 100:o + 140] = 3  # a poly-T run outside the masks
        mask.append([(600, 700)] if i % 2 == 0 else [(int(A.rlen[i]) - 50, int(A.rlen[i]))])
    A.mask = mask
    p = oracle.make_params(A.freq, k=k)
    ctx = _ctx(mb, A, k=k)
    ctx.load_block(0, A)
    n = ctx.sort_kmers(0)
    gc, gr, gp = ctx.get_kmers(0, n)
    oc, orr, op = oracle.sort_kmers(A, p)
    assert (oc == (1 << (2 * k)) - 1).sum() > 1000
    assert n == oc.size and (gc == oc).all() and (gr == orr).all() and (gp == op).all()
    ctx.close()


def test_masked_index_matches_oracle(mb):
    """-m track masking in tuple extraction (dalign/filter.c:428-470), masks mirrored for cB."""
    import oracle
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    rng = np.random.default_rng(3)
    mask = []
    for i in range(A.nreads):
        L = int(A.rlen[i])
        cuts = np.sort(rng.choice(L, size=2 * int(rng.integers(0, 4)), replace=False)).tolist()
        iv = [(cuts[j], cuts[j + 1]) for j in range(0, len(cuts), 2)]
        if i % 7 == 0:
            iv = [(0, 30)] + [x for x in iv if x[0] > 30]
        mask.append(iv)
    A.mask = mask
    p = oracle.make_params(A.freq)
    ctx = _ctx(mb, A)
    ctx.load_block(0, A)
    n = ctx.sort_kmers(0)
    gc, gr, gp = ctx.get_kmers(0, n)
    oc, orr, op = oracle.sort_kmers(A, p)
    assert n == oc.size and (gc == oc).all() and (gr == orr).all() and (gp == op).all()
    # the device complement mirrors the intervals like complement_DB
    ctx.complement_block(0, 2)
    n2 = ctx.sort_kmers(2)
    c2, r2, p2 = ctx.get_kmers(2, n2)
    oc2, or2, op2 = oracle.sort_kmers(dazzdb.complement_block(A), p)
    assert n2 == oc2.size and (c2 == oc2).all() and (r2 == or2).all() and (p2 == op2).all()
    # and the full masked comparison equals the oracle's
    import oracle as O
    recs, traces, _ = O.daligner(A, A, dazzdb.complement_block(A), p, True)
    ctx.reset_overlap_buffer()
    ctx.match_filter(0, 0, 1)
    ctx.match_filter(2, 1, 1)
    r, tr = ctx.overlaps()
    assert r.size == len(recs)
    for x, y, t in zip(r, recs, traces):
        for f in ("aread", "bread", "flags", "abpos", "aepos", "bbpos", "bepos", "diffs", "tlen"):
            assert int(x[f]) == int(y[f]), f
        assert (tr[int(x["toff"]):int(x["toff"]) + int(x["tlen"])] == t).all()
    ctx.close()


@pytest.mark.parametrize("comp", [0, 1])
def test_local_alignment_batch_matches_oracle(mb, comp):
    """Single Local_Alignment calls from seeds on real hits (and, for comp=1, from the same
    points on the complemented read: mostly dead starts that exercise the boundary logic)."""
    import oracle
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    B = dazzdb.complement_block(A) if comp else A
    p = oracle.make_params(A.freq)
    h, _ = oracle.match_hits(A, A, p, True)
    rng = np.random.default_rng(11 + comp)
    rows = h[rng.choice(len(h), size=600, replace=False)]
    diag, apos, ar, br = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3]
    anti = 2 * apos - diag
    aoff, boff = A.boff[ar] + 1, B.boff[br] + 1
    alen, blen = A.rlen[ar], B.rlen[br]
    ctx = _ctx(mb, A)
    out, tr, cells = ctx.local_alignment_batch(A.bases, aoff, alen, B.bases, boff, blen, diag, anti, comp)
    half = tr.shape[1] // 2
    for i in range(len(diag)):
        a = A.bases[aoff[i] - 1:aoff[i] + alen[i] + 1]
        b = B.bases[boff[i] - 1:boff[i] + blen[i] + 1]
        o, at, bt, oc = oracle.local_alignment(a, b, comp, int(diag[i]), int(anti[i]), p)
        assert (out[i] == o).all(), (i, out[i], o)
        assert (tr[i, :o[5]] == at).all() and (tr[i, half:half + o[11]] == bt).all()
        assert cells[i] == oc
    ctx.close()


def test_full_block_cfg1_matches_oracle_and_is_deterministic(mb, tmp_path):
    """The 1 Mbp / 20x workload (2.5k reads, 21 Mbp) end to end against the oracle, also
    with many pair groups routed through the wide-band kernel."""
    import oracle
    reads, _ = synth.generate("cfg1")
    dazzdb.write_db(str(tmp_path / "C"), reads, 200)
    A = dazzdb.open_block(str(tmp_path / "C.1"))
    ctx = mb.Context()
    r1, t1 = mb.daligner_block(ctx, A)
    r2, t2 = mb.daligner_block(ctx, A)
    assert (r1 == r2).all() and (t1 == t2).all()
    st = ctx.stats()
    # pair groups whose band outgrows 32 diagonals handed to the wide kernel: same output,
    # same seeds and cells
    ctx.set_wave_limit(32)
    r3, t3 = mb.daligner_block(ctx, A)
    st3 = ctx.stats()
    ctx.close()
    assert sum(st3["wide"]) > 100 and sum(st["wide"]) == 0
    assert (r3 == r1).all() and (t3 == t1).all()
    assert st3["seeds"] == st["seeds"] and st3["cells"] == st["cells"]
    recs, traces, ost = oracle.daligner(A, A, dazzdb.complement_block(A), oracle.make_params(A.freq), True)
    assert r1.size == len(recs)
    assert st["seeds"] == [ost["seeds_n"], ost["seeds_c"]]
    assert sum(st["cells"]) == ost["cells"]
    mb.write_las(str(tmp_path / "g.las"), r1, t1, 100)
    oracle.write_las(str(tmp_path / "o.las"), recs, traces, 100)
    ok, msg = dazzdb.las_equal(str(tmp_path / "g.las"), str(tmp_path / "o.las"))
    assert ok, msg


def test_context_reuse_across_blocks_matches_fresh_contexts(mb, tmp_path):
    """One context over blocks of different maximum read lengths (the aligner's scratch
    layout moves with maxlen) gives every block exactly the output of a fresh context."""
    blocks = []
    for name in ("cfg1", "tiny", "tiny_tandem"):
        reads, _ = synth.generate(name)
        dazzdb.write_db(str(tmp_path / name), reads, 200)
        blocks.append(dazzdb.open_block(str(tmp_path / (name + ".1"))))
    assert len({A.maxlen for A in blocks}) == 3
    ctx = mb.Context()
    seq = blocks + [blocks[0], blocks[2], blocks[1]]
    shared = [mb.daligner_block(ctx, A) for A in seq]
    ctx.close()
    for A, (r, t) in zip(seq, shared):
        f = mb.Context()
        r0, t0 = mb.daligner_block(f, A)
        f.close()
        assert r.size == r0.size and (r == r0).all() and (t == t0).all()


def test_size_independent_properties_cfg2(mb, tmp_path):
    """The bacterial workload at full size (~115 Mbp block): the output is sorted by
    (aread, bread, comp, abpos), every A-path has its B-path mirror, traces are consistent
    (Check_Trace_Points, dalign/align.c:3419-3449), and two runs are identical."""
    import bench
    A = dazzdb.open_block(bench.make_db("cfg2"))
    ctx = mb.Context()
    r, t = mb.daligner_block(ctx, A)
    r2, t2 = mb.daligner_block(ctx, A)
    ctx.close()
    assert (r == r2).all() and (t == t2).all()
    key = np.stack([r["aread"], r["bread"], r["flags"] & 1, r["abpos"]], 1)
    srt = key[np.lexsort(key.T[::-1])]
    assert (key == srt).all()
    # symmetric: an A-path (ar, br) record has a B-path (br, ar) record of the same orientation
    fwd = set(zip(r["aread"].tolist(), r["bread"].tolist(), (r["flags"] & 1).tolist()))
    assert all((b, a, c) in fwd for (a, b, c) in fwd)
    # trace points: pairs, sum of b deltas = b span, one pair per trace interval of a
    for i in range(0, r.size, 97):
        x = r[i]
        tr = t[int(x["toff"]):int(x["toff"]) + int(x["tlen"])]
        assert int(x["tlen"]) % 2 == 0
        assert int(tr[1::2].sum()) == int(x["bepos"] - x["bbpos"])
        npts = (int(x["aepos"]) - 1) // 100 - int(x["abpos"]) // 100 + 1
        assert int(x["tlen"]) == 2 * npts


@pytest.mark.parametrize("name", cases())
def test_compute_trace_pts_matches_reference(mb, name):
    """Compute_Trace_PTS (dalign/align.c:5286-5397) on the device: exact diffs of every
    record of every reference .las file of the goldens, against the diffs the reference's
    own Compute_Trace_PTS computes (tests/golden/trace_pts.npz, from
    tests/golden/make_trace_pts_golden.py).  The whole DB sits in one slot, its complement
    in another."""
    fx = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "trace_pts.npz"))
    d, meta = load(name)
    G = dazzdb.open_block(os.path.join(d, "G"))
    ctx = mb.Context()
    for las in meta["las"]:
        ts, recs, traces = dazzdb.read_las(os.path.join(d, las))
        tb = 1 if ts <= 125 else 2
        rec = np.zeros(recs.size, mb.OVL_DTYPE)
        for f in ("tlen", "diffs", "abpos", "bbpos", "aepos", "bepos", "flags", "aread", "bread"):
            rec[f] = recs[f]
        offs = np.cumsum([0] + [t.size * tb for t in traces])
        rec["toff"] = offs[:-1]
        tr = np.concatenate([t.view(np.uint8) if tb == 2 else t for t in traces]) if traces else np.zeros(1, np.uint8)
        ctx.new_align_spec(0.70, ts, G.freq)
        ctx.load_block(0, G)
        ctx.complement_block(0, 2)
        g = ctx.compute_trace_pts(rec, tr, 0, 0, 2)
        want = fx[f"{name}/{las}"]
        bad = np.nonzero(g != want)[0]
        assert bad.size == 0, (las, int(bad[0]), int(g[bad[0]]), int(want[bad[0]]))
    ctx.close()


@pytest.mark.parametrize("name", cases())
def test_duo_instance_matches_reference_golden(mb, name, tmp_path):
    """Every pair group on the duo instance (two 16-lane teams per warp, each with its own
    pair group, 64-diagonal rings; wider bands go to the wide instance): the reference's
    .las files."""
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu",
                             ctx_hook=lambda ctx: ctx.set_align_schedule([], [2]))
    assert sorted(names) == sorted(meta["las"])
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.parametrize("name,kinds", [("self_long_panels", None), ("self_default", None),
                                        ("self_long_panels", [1, 1, 0, 0, 0]), ("self_default", [0, 0, 1, 0, 1]),
                                        ("self_long_panels", [1, 2, 0, 2, 2]), ("self_default", [2, 0, 2, 1, 2])])
def test_length_class_schedule_gives_the_same_output(mb, name, kinds, tmp_path):
    """One aligner launch per length class (gd_set_align_schedule) instead of the one
    persistent launch, some classes on the wide instance: the same .las files."""
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu",
                             ctx_hook=lambda ctx: ctx.set_align_schedule([8000, 20000, 60000, 150000], kinds))
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


def test_get_overlaps_copies_whole_buffer_or_the_leading_records_that_fit(mb):
    """gd_get_overlaps with room for everything copies the whole sorted buffer; with fewer
    record slots or trace bytes it copies the leading records whose traces fit, and their
    traces, unchanged."""
    d, meta = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = _ctx(mb, A)
    mb.daligner_block(ctx, A)
    n, tb = ctx.sort_overlaps()
    assert n > 10 and tb > 0
    L = mb.lib()
    full_r = np.zeros(n, mb.OVL_DTYPE)
    full_t = np.zeros(tb, np.uint8)
    assert L.gd_get_overlaps(ctx.h, full_r.ctypes.data, full_t.ctypes.data, n, tb) == n
    bpt = 1  # -s100: one byte per trace value
    ends = full_r["toff"].astype(np.int64) + full_r["tlen"].astype(np.int64) * bpt
    assert ends[-1] == tb
    for rcap, tcap in ((n // 2, tb), (n, tb // 2), (n // 3, tb // 3)):
        want = int(min(rcap, np.searchsorted(ends, tcap, side="right")))
        r = np.zeros(max(rcap, 1), mb.OVL_DTYPE)
        t = np.zeros(max(tcap, 1), np.uint8)
        k = L.gd_get_overlaps(ctx.h, r.ctypes.data, t.ctypes.data, rcap, tcap)
        assert k == want
        assert (r[:k] == full_r[:k]).all()
        used = int(ends[k - 1]) if k else 0
        assert (t[:used] == full_t[:used]).all()
    ctx.close()

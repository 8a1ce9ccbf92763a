"""The allocation-free Local_Alignment entry point (gd_local_alignment_batch_noalloc).

It serves callers that cannot allocate device memory once they run -- an application that
hands all of HBM to its own pool, or a latency-critical loop where cudaMalloc's implicit
synchronization is not allowed.  Through the C ABI, it must return exactly what the
allocating entry point (gd_local_alignment_batch) returns, on two calls in a row (the
second call reuses the static scratch the first one left behind), and what the oracle's
Local_Alignment returns.  On long reads it must either agree or fail with the documented
error.  This file is collected last so that a failure here stops a -x run only after every
other test has run."""
import os

import numpy as np
import pytest

from golden_cases import load
from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu

PAD = 64


def _seeds(A, B, n, seed):
    import oracle
    h, _ = oracle.match_hits(A, A, oracle.make_params(A.freq), True)
    rng = np.random.default_rng(seed)
    rows = h[rng.choice(len(h), size=min(n, len(h)), replace=False)]
    diag, apos, ar, br = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3]
    return (A.boff[ar] + 1, A.rlen[ar], B.boff[br] + 1, B.rlen[br], diag.astype(np.int32),
            (2 * apos - diag).astype(np.int32))


def _noalloc(ctx, A, B, seeds, comp, trstride):
    """One call of the entry point on caller-owned device buffers; returns (rc, error,
    out12, traces, cells)."""
    import torch
    import marvel_b200 as mb
    L = mb.lib()
    dev = torch.device("cuda")
    aoff, alen, boff, blen, diag, anti = seeds
    # sequences get 64 bytes of slack before and after
    da = torch.full((A.bases.size + 2 * PAD,), 4, dtype=torch.uint8, device=dev)
    db = torch.full((B.bases.size + 2 * PAD,), 4, dtype=torch.uint8, device=dev)
    da[PAD:PAD + A.bases.size] = torch.from_numpy(A.bases).to(dev)
    db[PAD:PAD + B.bases.size] = torch.from_numpy(B.bases).to(dev)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(aoff=aoff.astype(np.int64), alen=alen.astype(np.int32), boff=boff.astype(np.int64),
              blen=blen.astype(np.int32), diag=diag, anti=anti).items()}
    out = torch.full((len(diag), 12), -7, dtype=torch.int32, device=dev)
    tr = torch.zeros((len(diag), trstride), dtype=torch.int16, device=dev)
    cells = torch.zeros(len(diag), dtype=torch.int64, device=dev)
    maxlen = int(max(alen.max(), blen.max()))
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.gd_local_alignment_batch_noalloc(ctx.h, da.data_ptr() + PAD, db.data_ptr() + PAD, t["aoff"].data_ptr(),
                                            t["alen"].data_ptr(), t["boff"].data_ptr(), t["blen"].data_ptr(),
                                            t["diag"].data_ptr(), t["anti"].data_ptr(), len(diag), maxlen, comp,
                                            out.data_ptr(), tr.data_ptr(), trstride, cells.data_ptr(), stream)
    torch.cuda.synchronize()
    err = L.gd_last_error().decode() if rc else ""
    return rc, err, out.cpu().numpy(), tr.cpu().numpy().view(np.uint16), cells.cpu().numpy()


def _same(o, g, cells, ref_out, ref_tr, ref_cells, trstride, tag):
    assert (o == ref_out).all(), f"{tag}: paths differ"
    half = trstride // 2
    for i in range(len(o)):
        assert (g[i, :o[i, 5]] == ref_tr[i, :o[i, 5]]).all(), f"{tag}: A trace of seed {i}"
        assert (g[i, half:half + o[i, 11]] == ref_tr[i, half:half + o[i, 11]]).all(), f"{tag}: B trace of seed {i}"
    assert (cells == ref_cells).all(), f"{tag}: cells"


def test_noalloc_matches_allocating_entry_point_and_oracle_twice():
    import torch
    import marvel_b200 as mb
    import oracle
    assert torch.cuda.is_available()
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.new_align_spec(0.70, 100, A.freq)   # set-up may allocate; the batch calls below do not
    p = oracle.make_params(A.freq)
    for call, (comp, seed) in enumerate([(0, 21), (1, 22)]):
        B = dazzdb.complement_block(A) if comp else A
        seeds = _seeds(A, B, 300, seed)
        ref_out, ref_tr, ref_cells = ctx.local_alignment_batch(A.bases, *seeds[:2], B.bases, *seeds[2:], comp)
        trstride = ref_tr.shape[1]
        rc, err, o, g, cells = _noalloc(ctx, A, B, seeds, comp, trstride)
        assert rc == 0, err
        _same(o, g, cells, ref_out, ref_tr, ref_cells, trstride, f"call {call}")
        # the oracle's Local_Alignment on every 10th seed (reads with their 4s on both sides)
        aoff, alen, boff, blen, diag, anti = seeds
        half = trstride // 2
        for i in range(0, len(diag), 10):
            a = A.bases[aoff[i] - 1:aoff[i] + alen[i] + 1]
            b = B.bases[boff[i] - 1:boff[i] + blen[i] + 1]
            oo, at, bt, oc = oracle.local_alignment(a, b, comp, int(diag[i]), int(anti[i]), p)
            assert (o[i] == oo).all(), f"call {call}, seed {i}: path differs from the oracle"
            assert (g[i, :o[i, 5]] == at).all() and (g[i, half:half + o[i, 11]] == bt).all()
            assert cells[i] == oc
    ctx.close()


def test_noalloc_long_reads_agree_or_name_the_seed():
    """Reads of 30-150 kbp: the pebble store bounds how wide a band may grow over a long
    alignment, so each batch either equals the allocating entry point or fails with the
    documented pebble error."""
    import marvel_b200 as mb
    d, _ = load("self_long_panels")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.new_align_spec(0.70, 100, A.freq)
    for comp, seed in ((0, 31), (1, 32)):
        B = dazzdb.complement_block(A) if comp else A
        seeds = _seeds(A, B, 96, seed)
        ref_out, ref_tr, ref_cells = ctx.local_alignment_batch(A.bases, *seeds[:2], B.bases, *seeds[2:], comp)
        trstride = ref_tr.shape[1]
        rc, err, o, g, cells = _noalloc(ctx, A, B, seeds, comp, trstride)
        if rc:
            assert "pebbles" in err, err
        else:
            _same(o, g, cells, ref_out, ref_tr, ref_cells, trstride, f"long reads, comp {comp}")
    ctx.close()


def test_noalloc_short_trace_stride_is_an_error():
    import marvel_b200 as mb
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.new_align_spec(0.70, 100, A.freq)
    seeds = _seeds(A, A, 64, 41)
    ref_out, _, _ = ctx.local_alignment_batch(A.bases, *seeds[:2], A.bases, *seeds[2:], 0)
    longest = int(max(ref_out[:, 5].max(), ref_out[:, 11].max()))
    assert longest > 4
    rc, err, _, _, _ = _noalloc(ctx, A, A, seeds, 0, 2 * (longest - 1))
    assert rc == -1 and "trstride" in err, err
    ctx.close()


def test_noalloc_rejects_reads_beyond_its_static_scratch():
    import marvel_b200 as mb
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.new_align_spec(0.70, 100, A.freq)
    L = mb.lib()
    rc = L.gd_local_alignment_batch_noalloc(ctx.h, None, None, None, None, None, None, None, None, 1, 300000, 0,
                                            None, None, 64, None, None)
    assert rc == -1 and b"exceed" in L.gd_last_error()
    ctx.close()

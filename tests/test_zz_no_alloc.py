"""The allocation-free Local_Alignment entry point (gd_local_alignment_batch_noalloc).

It serves callers that cannot allocate device memory once they run -- an application that
hands all of HBM to its own pool, or a latency-critical loop where cudaMalloc's implicit
synchronization is not allowed.  Through the C ABI, it must return exactly what the
allocating entry point (gd_local_alignment_batch) returns, on two calls in a row (the
second call reuses the static scratch the first one left behind).  This file is collected
last so that a failure here stops a -x run only after every other test has run."""
import os

import numpy as np
import pytest

from golden_cases import load
from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu


def _seeds(A, B, n, seed):
    import oracle
    h, _ = oracle.match_hits(A, A, oracle.make_params(A.freq), True)
    rng = np.random.default_rng(seed)
    rows = h[rng.choice(len(h), size=n, replace=False)]
    diag, apos, ar, br = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3]
    return (A.boff[ar] + 1, A.rlen[ar], B.boff[br] + 1, B.rlen[br], diag.astype(np.int32),
            (2 * apos - diag).astype(np.int32))


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import marvel_b200 as mb
    assert torch.cuda.is_available()
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.new_align_spec(0.70, 100, A.freq)   # set-up may allocate; the batch calls below do not
    L = mb.lib()
    dev = torch.device("cuda")
    pad = 64
    for call, (comp, seed) in enumerate([(0, 21), (1, 22)]):
        B = dazzdb.complement_block(A) if comp else A
        aoff, alen, boff, blen, diag, anti = _seeds(A, B, 300, seed)
        ref_out, ref_tr, ref_cells = ctx.local_alignment_batch(A.bases, aoff, alen, B.bases, boff, blen, diag, anti,
                                                               comp)
        trstride = ref_tr.shape[1]
        # caller-owned device buffers; sequences get 64 bytes of slack before and after
        da = torch.full((A.bases.size + 2 * pad,), 4, dtype=torch.uint8, device=dev)
        db = torch.full((B.bases.size + 2 * pad,), 4, dtype=torch.uint8, device=dev)
        da[pad:pad + A.bases.size] = torch.from_numpy(A.bases).to(dev)
        db[pad:pad + B.bases.size] = torch.from_numpy(B.bases).to(dev)
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
             dict(aoff=aoff.astype(np.int64), alen=alen.astype(np.int32), boff=boff.astype(np.int64),
                  blen=blen.astype(np.int32), diag=diag, anti=anti).items()}
        out = torch.full((len(diag), 12), -7, dtype=torch.int32, device=dev)
        tr = torch.zeros((len(diag), trstride), dtype=torch.int16, device=dev)
        cells = torch.zeros(len(diag), dtype=torch.int64, device=dev)
        maxlen = int(max(alen.max(), blen.max()))
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.gd_local_alignment_batch_noalloc(ctx.h, da.data_ptr() + pad, db.data_ptr() + pad,
                                                t["aoff"].data_ptr(), t["alen"].data_ptr(), t["boff"].data_ptr(),
                                                t["blen"].data_ptr(), t["diag"].data_ptr(), t["anti"].data_ptr(),
                                                len(diag), maxlen, comp, out.data_ptr(), tr.data_ptr(), trstride,
                                                cells.data_ptr(), stream)
        assert rc == 0, L.gd_last_error().decode()
        torch.cuda.synchronize()
        o = out.cpu().numpy()
        assert (o == ref_out).all(), f"call {call}: paths differ"
        half = trstride // 2
        g = tr.cpu().numpy().view(np.uint16)
        for i in range(len(diag)):
            assert (g[i, :o[i, 5]] == ref_tr[i, :o[i, 5]]).all()
            assert (g[i, half:half + o[i, 11]] == ref_tr[i, half:half + o[i, 11]]).all()
        assert (cells.cpu().numpy() == ref_cells).all()
    ctx.close()


def test_noalloc_rejects_reads_beyond_its_static_scratch():
    import marvel_b200 as mb
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.new_align_spec(0.70, 100, A.freq)
    L = mb.lib()
    rc = L.gd_local_alignment_batch_noalloc(ctx.h, None, None, None, None, None, None, None, None, 1, 200000, 0,
                                            None, None, 64, None, None)
    assert rc == -1 and b"exceed" in L.gd_last_error()
    ctx.close()

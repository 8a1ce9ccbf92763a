"""Learned triage of pair groups: the BF16 tensor-core MLP kernels against the float64
restatement (tests/mlp_ref.py), the device training loop, and the triaged pipeline: every
record it emits is a plain-path record, record recall >= 99.5 % on a genome the model was
not trained on, and fewer wave cells than the plain path."""
import numpy as np
import pytest

import mlp_ref
from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


def _random_model(rng, n=2000):
    from marvel_b200 import triage
    x = rng.normal(size=(n, 12)).astype(np.float32) * rng.uniform(0.5, 4, 12).astype(np.float32) + \
        rng.normal(size=12).astype(np.float32)
    p = triage.mlp_init(x, seed=7)
    p[mlp_ref.OFF_B1:mlp_ref.OFF_W2] = rng.normal(scale=0.1, size=64)
    p[mlp_ref.OFF_B2:mlp_ref.OFF_W3] = rng.normal(scale=0.1, size=64)
    p[mlp_ref.OFF_B3] = 0.3
    return x, p


def test_mlp_forward_matches_reference(mb):
    """Forward on tensor cores vs float64 with the kernel's bf16 roundings emulated
    (tolerance 2e-3 absolute on p) and vs plain float64 (tolerance 3e-2 absolute)."""
    rng = np.random.default_rng(1)
    x, p = _random_model(rng, 1000)
    ctx = mb.Context()
    pg = ctx.mlp_forward(p, x[:999])
    ctx.close()
    pe = mlp_ref.prob(p, x[:999], emulate_bf16=True)
    pf = mlp_ref.prob(p, x[:999])
    assert np.abs(pg - pe).max() < 2e-3
    assert np.abs(pg - pf).max() < 3e-2


@pytest.mark.parametrize("n,pos_weight", [(64, 1.0), (300, 1.0), (4096, 5.0)])
def test_mlp_gradient_matches_reference(mb, n, pos_weight):
    """Backward (dW2, dH1, dW1 as tensor-core GEMMs over the batch, biases and the last
    layer in FP32) against (a) the float64 gradient with the kernels' bf16 roundings
    emulated: relative L2 error < 1e-2 per layer; (b) the plain float64 gradient: cosine
    > 0.999 and relative L2 error < 3e-2 over all trained parameters.  Loss within 1e-3."""
    rng = np.random.default_rng(n)
    x, p = _random_model(rng, n)
    y = (rng.random(n) < 0.3).astype(np.float32)
    ctx = mb.Context()
    g, loss = ctx.mlp_grad(p, x, y, pos_weight)
    ctx.close()
    lr, gr = mlp_ref.loss_grad(p, x, y, pos_weight)
    le, ge = mlp_ref.loss_grad_bf16(p, x, y, pos_weight)
    assert abs(loss - le) <= 1e-3 * abs(le)
    assert abs(loss - lr) <= 1e-2 * abs(lr)
    assert np.all(g[:mlp_ref.OFF_W1] == 0)
    a, b = g[mlp_ref.OFF_W1:].astype(np.float64), gr[mlp_ref.OFF_W1:]
    assert a @ b / (np.linalg.norm(a) * np.linalg.norm(b)) > 0.999
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 3e-2
    for lo, hi in ((mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
                   (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.NPARAM)):
        assert np.linalg.norm(g[lo:hi] - ge[lo:hi]) <= 1e-2 * np.linalg.norm(ge[lo:hi]) + 1e-8, (lo, hi)


def test_mlp_training_learns_a_separable_rule(mb):
    """The device Adam loop drives the loss down and fits a nonlinear rule."""
    from marvel_b200 import triage
    rng = np.random.default_rng(3)
    x = rng.normal(size=(20000, 12)).astype(np.float32)
    y = ((x[:, 0] * x[:, 1] > 0) & (x[:, 2] > -1)).astype(np.float32)
    ctx = mb.Context()
    p0 = triage.mlp_init(x, seed=1)
    p, losses = ctx.mlp_train(x, y, p0, epochs=15, batch=1024, lr=3e-3, seed=1)
    prob = ctx.mlp_forward(p, x)
    ctx.close()
    assert losses[-1] < 0.5 * losses[0]
    assert np.all(p[:24] == p0[:24])   # the feature scales are not trained
    assert ((prob > 0.5) == (y > 0.5)).mean() > 0.95


def _workload_db(seed_offset, scale):
    import bench
    return dazzdb.open_block(bench.make_db("cfg2", seed_offset=seed_offset, scale=scale))


def _collect(mb, ctx, A):
    ctx.triage_reset()
    ctx.triage_collect(True)
    r, t = mb.daligner_block(ctx, A)
    ctx.triage_collect(False)
    feat, rec, cells = ctx.triage_groups()
    return r, t, feat, rec, cells


def test_triage_keeps_recall_and_saves_cells(mb):
    """Train on one genome (the bacterial workload's shape at 1/4 size), apply to another
    (different seed): the triaged records are a subset of the plain ones, record recall is
    >= 99.5 %, and the aligner computes fewer wave cells."""
    from marvel_b200 import triage
    ctx = mb.Context()
    _, _, feat, rec, cells = _collect(mb, ctx, _workload_db(0, 0.25))
    assert feat.shape[0] == rec.size > 1000 and (cells > 0).any()
    st = ctx.stats()
    assert int(rec.sum()) == st["records"]   # per-group records add up to the buffer
    model, info = triage.fit(ctx, feat, rec, recall=0.999, epochs=25)
    assert info["losses"][-1] < info["losses"][0]

    B = _workload_db(1, 0.25)
    rp, tp, featb, recb, cellsb = _collect(mb, ctx, B)
    plain_cells = sum(ctx.stats()["cells"])
    ctx.triage_set_model(model.params, model.threshold)
    rt, tt = mb.daligner_block(ctx, B)
    st = ctx.stats()
    ctx.triage_set_model(None)
    ctx.close()
    # every triaged record (with its trace) is a plain record
    def keyed(r, t):
        out = {}
        for x in r:
            o = int(x["toff"])
            out[(int(x["aread"]), int(x["bread"]), int(x["flags"]) & 1, int(x["abpos"]), int(x["aepos"]),
                 int(x["bbpos"]), int(x["bepos"]), int(x["diffs"]))] = t[o:o + int(x["tlen"])].tobytes()
        return out
    kp, kt = keyed(rp, tp), keyed(rt, tt)
    assert all(k in kp and kp[k] == v for k, v in kt.items())
    recall = len(kt) / len(kp)
    assert recall >= 0.995, recall
    assert sum(st["skipped"]) > 0
    assert sum(st["cells"]) < plain_cells
    # the device skip decision agrees with the model evaluated on the collected features
    pb = mb.Context().mlp_forward(model.params, featb)
    ev = triage.evaluate(pb, recb, cellsb, model.threshold)
    assert abs(ev["groups_skipped"] * featb.shape[0] - sum(st["skipped"])) <= 0.001 * featb.shape[0] + 2


def _features_f64(hits, rlen_a, rlen_b, binshift, minover, minhit, comp):
    """The 12 features of every pair group of >= minhit hits, restated in float64 from the
    sorted hit list (rows diag, apos, aread, bread): {(n, alen, blen): [feature rows]}."""
    d, ap, ar, br = (hits[:, i].astype(np.int64) for i in range(4))
    cut = np.flatnonzero((np.diff(ar) != 0) | (np.diff(br) != 0)) + 1
    starts = np.concatenate([[0], cut])
    ends = np.concatenate([cut, [d.size]])
    out = {}
    for s, e in zip(starts, ends):
        n = e - s
        if n < minhit:
            continue
        dd = d[s:e].astype(np.float64)
        alen, blen = float(rlen_a[ar[s]]), float(rlen_b[br[s]])
        mean = dd.sum() / n
        var = max((dd * dd).sum() / n - mean * mean, 0.0)
        near = np.count_nonzero(np.abs(dd - mean) <= (1 << binshift))
        ovl = min(alen, blen + mean) - max(0.0, mean)
        span = float(ap[e - 1] - ap[s])
        f = [np.log2(n), np.log2(alen), np.log2(blen), span / alen, np.log2(1 + d[s:e].max() - d[s:e].min()),
             mean / alen, np.log2(1 + np.sqrt(var)), ovl / (2.0 * minover), 64.0 * n / (span + 1), near / n,
             float(comp), 0.0]
        out.setdefault((n, int(alen), int(blen)), []).append(np.array(f))
    return out


def test_group_features_equal_a_float64_restatement(mb):
    """The features the fused selection computes -- by one thread for short groups and by a
    warp for groups of more than 32 hits -- equal a float64 restatement from the sorted hits
    (to float32 rounding and the device's log2f)."""
    import os
    from golden_cases import load
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.set_filter_params(14, 6, 0, 35)
    ctx.new_align_spec(0.70, 100, A.freq)
    ctx.set_globals(2000, False, 32 << 30)
    ctx.load_block(0, A)
    ctx.sort_kmers(0)
    ctx.triage_reset()
    ctx.triage_collect(True)
    ctx.match_filter(0, 0, 1)
    ctx.triage_collect(False)
    feat, rec, cells = ctx.triage_groups()
    hits = ctx.get_hits()
    ctx.close()
    # binshift 6 (-w6), minover 2000 (the context's global: 2 x -l1000), minhit 3 (-h35, -k14)
    ref = _features_f64(hits, A.rlen, A.rlen, 6, 2000, 3, 0)
    assert feat.shape[0] > 100
    n = np.rint(np.exp2(feat[:, 0].astype(np.float64))).astype(np.int64)
    assert (n > 32).sum() > 10, "the case should hold groups long enough for the warp path"
    for row, ni in zip(feat, n):
        key = (int(ni), int(round(2.0 ** float(row[1]))), int(round(2.0 ** float(row[2]))))
        cands = ref.get(key, [])
        assert any(np.allclose(row, c, rtol=2e-6, atol=2e-6) for c in cands), (key, row, cands[:2])


def test_duo_instance_honours_the_skip_flags(mb):
    """The triage's skip flags reach the duo aligner instance as they reach the warp instance:
    the same groups skipped and the same records (a random model, thresholded at the median of
    its outputs so that about half the groups are skipped)."""
    import os
    from golden_cases import load
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    rng = np.random.default_rng(11)
    _, params = _random_model(rng)

    def ctx_for(kinds):
        ctx = mb.Context()
        ctx.set_filter_params(14, 6, 0, 35)
        ctx.new_align_spec(0.70, 100, A.freq)
        ctx.set_globals(2000, False, 32 << 30)
        if kinds is not None:
            ctx.set_align_schedule([], kinds)
        return ctx

    ctx = ctx_for(None)
    _, _, feat, _, _ = _collect(mb, ctx, A)
    thr = float(np.median(ctx.mlp_forward(params, feat)))
    ctx.close()
    out = []
    for kinds in (None, [2]):
        ctx = ctx_for(kinds)
        ctx.triage_set_model(params, thr)
        r, t = mb.daligner_block(ctx, A)
        st = ctx.stats()
        out.append((dazzdb.las_digest(r, t, r["toff"], 1), sum(st["skipped"]), sum(st["cells"])))
        ctx.close()
    assert out[0][1] > 0
    assert out[0] == out[1]

"""The CPU restatement (oracle) reproduces the reference daligner's golden .las files."""
import os

import numpy as np

import pytest

import daligner_run
from golden_cases import cases, d2_cases, load
from marvel_b200 import dazzdb


@pytest.mark.parametrize("name", cases())
def test_oracle_matches_reference_golden(name, tmp_path):
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "oracle")
    assert sorted(names) == sorted(meta["las"])
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.parametrize("name", d2_cases())
def test_oracle_matches_reference_daligner2_golden(name, tmp_path):
    """The daligner2 restatement (modimizer index, one join for both orientations, its
    report and Handle_Redundancies) reproduces the reference daligner2's .las files."""
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "oracle", variant=2)
    assert sorted(names) == sorted(meta["las"])
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


def test_oracle_kmer_index_is_sorted_and_complete():
    import oracle
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    p = oracle.make_params(A.freq)
    code, read, rpos = oracle.sort_kmers(A, p)
    assert code.size == A.totlen - A.nreads * (14 - 1)
    key = (code.astype(object) << 64) | (read.astype(object) << 32) | rpos.astype(object)
    assert all(key[i] < key[i + 1] for i in range(0, code.size - 1, 997))
    # spot-check codes against the bases
    for i in range(0, code.size, 50021):
        s = A.read(int(read[i]))[int(rpos[i]) - 13:int(rpos[i]) + 1]
        c = 0
        for x in s:
            c = (c << 2) | int(x)
        assert c == int(code[i])


def test_oracle_hits_sorted_by_bread_aread_apos():
    import oracle
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    h, limit = oracle.match_hits(A, A, oracle.make_params(A.freq), True)
    assert limit == 10000
    k = list(zip(h[:, 3], h[:, 2], h[:, 1], -h[:, 0]))
    assert k == sorted(k)
    assert (h[:, 3] < h[:, 2]).all()   # within a block only b-read < a-read pairs


def test_oracle_d2_bridging_matches_reference():
    """daligner2's Handle_Redundancies with its bridging pass (Compute_Bridge_Path ->
    Compute_Alignment(DIFF_TRACE) -> trace_nd/split_nd, Bridge) against the reference's own
    function on the one-pair fixtures (tests/golden/make_d2_bridge_golden.py): paths kept,
    coordinates, diffs and every trace value."""
    import d2_bridge_cases as dbc
    cases, expected = dbc.load(os.path.join(os.path.dirname(__file__), "golden", "d2_bridge", "cases.npz"))
    bridged = 0
    for i, (c, (ea, eb)) in enumerate(zip(cases, expected)):
        ga, gb = dbc.oracle_run(c)
        assert [h for h, _ in ga] == [h for h, _ in ea], i
        assert all(np.array_equal(x, y) for (_, x), (_, y) in zip(ga, ea)), i
        if eb is not None:
            assert [h for h, _ in gb] == [h for h, _ in eb], i
            assert all(np.array_equal(x, y) for (_, x), (_, y) in zip(gb, eb)), i
        bridged += dbc.was_bridged(c, (ea, eb))
    assert bridged >= len(cases) // 2


def _trace_pts_fixture():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "trace_pts.npz"))


@pytest.mark.parametrize("name", cases())
def test_oracle_trace_pts_matches_reference_compute_trace_pts(name):
    """The restatement of Compute_Trace_PTS / iter_np (dalign/align.c:4556-4917, 5286-5397)
    gives, on every record of every golden .las file, the diffs the reference's own
    Compute_Trace_PTS computes (tests/golden/make_trace_pts_golden.py)."""
    import oracle
    fx = _trace_pts_fixture()
    d, meta = load(name)
    G = dazzdb.open_block(os.path.join(d, "G"))
    Gc = dazzdb.complement_block(G)
    for las in meta["las"]:
        ts, recs, traces = dazzdb.read_las(os.path.join(d, las))
        want = fx[f"{name}/{las}"]
        assert want.size == recs.size
        for i in range(recs.size):
            r = recs[i]
            bb = (Gc if r["flags"] & 1 else G).read(int(r["bread"]) - G.ufirst)
            got = oracle.trace_pts_diffs(G.read(int(r["aread"]) - G.ufirst), bb, r, traces[i], ts)
            assert got == int(want[i]), (las, i, got, int(want[i]))


def test_oracle_matches_reference_on_full_cfg1_block():
    """The restatement on the whole cfg1 block (1 Mbp genome, 20x; regenerated from its seed)
    gives the records the reference daligner writes for it (digest of the reference's
    .las, tests/golden/config_digests.json) and the reference's wave-cell count."""
    import json
    import oracle
    from marvel_b200 import synth
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_digests.json")) as f:
        want = json.load(f)["cfg1"]
    A = dazzdb.open_block(synth.cached_db(want["workload"], want["seed_offset"], want["scale"]))
    recs, traces, st = oracle.daligner(A, A, dazzdb.complement_block(A), oracle.make_params(A.freq), True)
    toff = np.zeros(len(traces), np.int64)
    if len(traces):
        toff[1:] = np.cumsum([t.size for t in traces])[:-1]
    tb = np.concatenate(traces).astype(np.uint8) if traces else np.zeros(0, np.uint8)
    digest, n = dazzdb.las_digest(recs, tb, toff, 1)
    assert n == want["novl"] and digest == want["sha256"]
    assert st["cells"] == want["cells"]

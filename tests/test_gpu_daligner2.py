"""GPU parity of the daligner2 (modimizer seeds, dalign2/) path: the reference daligner2's
golden .las files, its sorted index against the oracle, and a block pair the goldens do not
cover against the oracle.  Bit-exact (integer work)."""
import os

import numpy as np
import pytest

import daligner_run
from golden_cases import d2_cases, load
from marvel_b200 import dazzdb, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


@pytest.mark.parametrize("name", d2_cases())
def test_gpu_matches_reference_daligner2_golden(mb, name, tmp_path):
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu", variant=2)
    assert sorted(names) == sorted(meta["las"])
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.parametrize("name", ["d2_self", "d2_pair_dust"])
def test_duo_schedule_keeps_daligner2_on_the_warp_instance(mb, name, tmp_path):
    """daligner2's report has no duo instance: a schedule asking for it runs the warp instance
    in its place, and the .las files are still the reference's."""
    d, meta = load(name)
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu", variant=2,
                             ctx_hook=lambda ctx: ctx.set_align_schedule([], [2]))
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.parametrize("name,k,t", [("d2_self", 14, 0), ("d2_self_k16_w5", 16, 0), ("d2_self_asym_t20", 14, 20),
                                      ("d2_pair_dust", 14, 0)])
def test_d2_kmer_index_matches_oracle(mb, name, k, t):
    """Codes, (read << 1 | strand) and positions of the sorted index, entry for entry
    (masked reads included for the dust case)."""
    import oracle
    d, meta = load(name)
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    if any(f.startswith("-mdust") for f in meta["flags"]):
        dazzdb.load_track(A, "dust")
    p = oracle.make_params(A.freq, k=k, t=t, variant=2)
    code, read, rpos = oracle.sort_kmers2(A, p)
    assert code.size > 1000 and (read & 1).any() and not (read & 1).all()
    ctx = mb.Context()
    ctx.set_variant(2)
    ctx.set_filter_params(k, 6, t, 35)
    ctx.load_block(0, A)
    n = ctx.sort_kmers(0)
    gc, gr, gp = ctx.get_kmers(0, n)
    ctx.close()
    assert n == code.size
    assert np.array_equal(gc, code) and np.array_equal(gr, read) and np.array_equal(gp, rpos)


def test_d2_small_pair_matches_oracle(mb, tmp_path):
    """A two-block DB of the repeat-bearing small workload (not among the goldens): the GPU
    and the oracle write the same .las files, and both orientations find overlaps."""
    reads, _ = synth.generate("small", 0.5)
    dazzdb.write_db(str(tmp_path / "G"), reads, 0.6)
    flags = ["-M32", "-k14", "-w6", "-h35", "-e.70", "-l1000", "-s100"]
    go = daligner_run.run(str(tmp_path), flags, ["G.1", "G.2"], str(tmp_path / "o"), "oracle", variant=2)
    gg = daligner_run.run(str(tmp_path), flags, ["G.1", "G.2"], str(tmp_path / "g"), "gpu", variant=2)
    assert go == gg
    comp = 0
    for n in gg:
        ok, msg = dazzdb.las_equal(str(tmp_path / "g" / n), str(tmp_path / "o" / n))
        assert ok, f"{n}: {msg}"
        _, recs, _ = dazzdb.read_las(str(tmp_path / "g" / n))
        comp += int((recs["flags"] & 1).sum())
    assert comp > 0


def test_d2_stats_split_orientations(mb):
    """One join gives both orientations: hits and records in each, and the filter entry of the
    other mode is refused."""
    d, _ = load("d2_self")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    r, _ = mb.daligner2_block(ctx, A)
    st = ctx.stats()
    assert st["hits"][0] > 0 and st["hits"][1] > 0
    assert r.size > 0 and (r["flags"] & 1).any() and not (r["flags"] & 1).all()
    with pytest.raises(mb.GpuError):
        ctx.match_filter(0, 0, 1)
    ctx.close()


def test_d2_bridging_matches_reference(mb):
    """daligner2's Handle_Redundancies with its bridging pass on the device, one pair per call,
    against the reference's own function on the one-pair fixtures
    (tests/golden/make_d2_bridge_golden.py): paths kept, coordinates, diffs, trace values."""
    import d2_bridge_cases as dbc
    cases, expected = dbc.load(os.path.join(os.path.dirname(__file__), "golden", "d2_bridge", "cases.npz"))
    ctx = mb.Context()
    for i, (c, (ea, eb)) in enumerate(zip(cases, expected)):
        ps = c.amatch + (c.bmatch or [])
        hdr, tr = dbc.flat(ps)
        a = np.concatenate([[4], c.a, [4]]).astype(np.uint8)
        b = np.concatenate([[4], c.b, [4]]).astype(np.uint8)
        tcap = int(tr.size) + 8 * (max(c.a.size, c.b.size) // c.tspace + 8) * len(ps) + 1024
        n, oh, ot = ctx.test_handle_redundancies_d2(a, b, c.tspace, c.comp, hdr, tr, len(c.amatch),
                                                    c.bmatch is not None, tcap)
        want = ea + (eb or [])
        assert n == len(ea), i
        o = 0
        for j, (h, t) in enumerate(want):
            assert [int(x) for x in oh[j]] == h, (i, j)
            assert np.array_equal(ot[o:o + h[5]], t), (i, j)
            o += h[5]
    ctx.close()

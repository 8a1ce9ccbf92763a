"""Edge cases of a block comparison, the device path against the oracle: a block of one
read, reads of exactly k bases, blocks that share no k-mer (no hits, no pair groups),
homopolymer reads and tandem repeats (a few k-mers with long runs, which the pair cap of
-M trims).  Bit-exact: records, traces, seeds and wave cells."""
import numpy as np
import pytest

from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


def _block(reads):
    rlen = np.array([r.size for r in reads], np.int32)
    boff = np.zeros(len(reads) + 1, np.int64)
    boff[1:] = np.cumsum(rlen.astype(np.int64) + 1)
    bases = np.full(int(boff[-1]) + 1, 4, np.uint8)
    for i, r in enumerate(reads):
        bases[boff[i] + 1:boff[i] + 1 + r.size] = r
    return dazzdb.Block(bases=bases, boff=boff, rlen=rlen, ufirst=0, part=1,
                        freq=np.full(4, 0.25, np.float32), maxlen=int(rlen.max()), totlen=int(rlen.sum()))


def _cases():
    rng = np.random.default_rng(1)

    def rnd(n):
        return rng.integers(0, 4, n).astype(np.uint8)

    def noisy(s, rate):  # substitutions, insertions and deletions at rate
        out = []
        for b in s:
            r = rng.random()
            if r < rate / 3:
                continue
            if r < 2 * rate / 3:
                out.append(rng.integers(0, 4))
            elif r < rate:
                b = (b + rng.integers(1, 4)) % 4
            out.append(b)
        return np.array(out, np.uint8)

    g = rnd(20000)
    return {
        "one_read": ([noisy(g[:6000], 0.1)], None),
        "kmer_length_reads": ([rnd(14), noisy(g[:5000], 0.1), rnd(14), noisy(g[2000:7000], 0.1)], None),
        "no_shared_kmers": ([rnd(3000) for _ in range(3)], [rnd(3000) for _ in range(3)]),
        "homopolymer": ([np.zeros(1500, np.uint8), np.zeros(1200, np.uint8), noisy(g[:4000], 0.1),
                         noisy(g[1000:5000], 0.1)], None),
        "tandem_repeat": ([np.tile(rnd(7), 300), np.tile(rnd(7), 250), noisy(g[:3000], 0.05)], None),
    }


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_edge_case_matches_oracle(mb, name, tmp_path):
    import oracle
    ra, rb = CASES[name]
    A = _block(ra)
    B = _block(rb) if rb is not None else None
    ctx = mb.Context()
    recs, tr = mb.daligner_block(ctx, A, B, k=14, w=6, h=35, e=0.70, l=1000, s=100, M=32)
    st = ctx.stats()
    ctx.close()
    Bo = B if B is not None else A
    orecs, otraces, ost = oracle.daligner(A, Bo, dazzdb.complement_block(Bo), oracle.make_params(A.freq),
                                          B is None)
    assert recs.size == len(orecs), (name, recs.size, len(orecs))
    assert st["seeds"] == [ost["seeds_n"], ost["seeds_c"]]
    assert sum(st["cells"]) == ost["cells"]
    mb.write_las(str(tmp_path / "g.las"), recs, tr, 100)
    oracle.write_las(str(tmp_path / "o.las"), orecs, otraces, 100)
    ok, msg = dazzdb.las_equal(str(tmp_path / "g.las"), str(tmp_path / "o.las"))
    assert ok, f"{name}: {msg}"

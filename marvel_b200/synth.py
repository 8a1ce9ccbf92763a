"""Seeded synthetic genomes and long reads for the daligner workloads.

The reference ships no datasets for the overlap path, so every workload is generated
here from a seed with numpy's PCG64.  A workload is a genome model (random ACGT with
optional repeat families, a second haplotype, tandem repeats) plus a read model
(log-normal lengths, uniform start, random strand, i.i.d. insertion / deletion /
substitution errors with an optional homopolymer deletion bias).

Bases are encoded 0..3 = A,C,G,T exactly as the Dazzler DB stores them
(db/DB.c:261-309, Compress_Read / Uncompress_Read).
"""
from __future__ import annotations

import dataclasses
import numpy as np

__all__ = ["ReadModel", "GenomeModel", "Workload", "WORKLOADS", "make_genome", "make_reads", "generate"]


@dataclasses.dataclass(frozen=True)
class GenomeModel:
    length: int
    # (copies, unit length, divergence) triples inserted at random places
    repeats: tuple = ()
    # fraction of the genome covered by interspersed repeat families
    # (unit 1..10 kbp, divergence in [div_lo, div_hi])
    interspersed_frac: float = 0.0
    interspersed_len: tuple = (1000, 10000)
    interspersed_div: tuple = (0.05, 0.15)
    tandem_frac: float = 0.0
    tandem_period: tuple = (2, 201)
    diploid_snp: float = 0.0
    diploid_indel: float = 0.0
    # background base probabilities (A, C, G, T); empty = uniform
    base_probs: tuple = ()


@dataclasses.dataclass(frozen=True)
class ReadModel:
    coverage: float
    mean_len: float
    sd_len: float
    min_len: int = 1000
    max_len: int = 30000
    p_ins: float = 0.09
    p_del: float = 0.045
    p_sub: float = 0.015
    homopolymer_del_bias: float = 1.0  # deletion rate multiplier inside homopolymers >= 4


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    genome: GenomeModel
    reads: ReadModel
    seed: int
    # DB blocks (DBsplit -s<block_mbp>); 0 = the whole DB in one block.  nblocks > 0 generates
    # only the reads of the first nblocks blocks: the reads come in random genome order, so
    # these are exactly the first blocks of the full-coverage DB.
    block_mbp: float = 0
    nblocks: int = 0
    # interval tracks daligner masks with (-m), made by DBdust on the whole DB
    masks: tuple = ()


def _mutate_subs(rng, seq, rate):
    if rate <= 0:
        return seq
    seq = seq.copy()
    pos = np.nonzero(rng.random(seq.size) < rate)[0]
    seq[pos] = (seq[pos] + rng.integers(1, 4, pos.size, dtype=np.uint8)) & 3
    return seq


def _mutate_indels(rng, seq, rate):
    """Short (1-3 bp) insertions and deletions at the given per-base rate."""
    if rate <= 0:
        return seq
    ev = np.nonzero(rng.random(seq.size) < rate)[0]
    if ev.size == 0:
        return seq
    keep = np.ones(seq.size, dtype=bool)
    is_del = rng.random(ev.size) < 0.5
    lens = rng.integers(1, 4, ev.size)
    for p, d, l in zip(ev[is_del], is_del[is_del], lens[is_del]):
        keep[p:p + l] = False
    out = seq[keep]
    ins_at = np.sort(np.searchsorted(np.cumsum(keep) - 1, ev[~is_del]))
    ins_len = lens[~is_del]
    if ins_at.size:
        chunks = []
        prev = 0
        for a, l in zip(ins_at, ins_len):
            chunks.append(out[prev:a])
            chunks.append(rng.integers(0, 4, l, dtype=np.uint8))
            prev = a
        chunks.append(out[prev:])
        out = np.concatenate(chunks)
    return out


def make_genome(model: GenomeModel, rng: np.random.Generator):
    """Returns a list of haplotype arrays (uint8 0..3)."""
    if model.base_probs:
        g = rng.choice(4, size=model.length, p=np.asarray(model.base_probs, float)).astype(np.uint8)
    else:
        g = rng.integers(0, 4, model.length, dtype=np.uint8)
    n = model.length
    # fixed repeat families: copies of one unit at a given divergence
    for copies, unit, div in model.repeats:
        base = rng.integers(0, 4, unit, dtype=np.uint8)
        for _ in range(copies):
            p = int(rng.integers(0, n - unit))
            g[p:p + unit] = _mutate_subs(rng, base, div)
    if model.interspersed_frac > 0:
        target = int(model.interspersed_frac * n)
        covered = 0
        nfam = max(1, target // 200000)
        fams = [rng.integers(0, 4, int(rng.integers(*model.interspersed_len)), dtype=np.uint8)
                for _ in range(nfam)]
        while covered < target:
            f = fams[int(rng.integers(0, nfam))]
            div = float(rng.uniform(*model.interspersed_div))
            p = int(rng.integers(0, n - f.size))
            g[p:p + f.size] = _mutate_subs(rng, f, div)
            covered += f.size
    if model.tandem_frac > 0:
        target = int(model.tandem_frac * n)
        covered = 0
        while covered < target:
            period = int(rng.integers(*model.tandem_period))
            unit = rng.integers(0, 4, period, dtype=np.uint8)
            span = int(rng.integers(500, 5000))
            arr = np.tile(unit, span // period + 1)[:span]
            p = int(rng.integers(0, n - span))
            g[p:p + span] = _mutate_subs(rng, arr, 0.02)
            covered += span
    haps = [g]
    if model.diploid_snp > 0 or model.diploid_indel > 0:
        h2 = _mutate_subs(rng, g, model.diploid_snp)
        h2 = _mutate_indels(rng, h2, model.diploid_indel)
        haps.append(h2)
    return haps


def _lognormal_params(mean, sd):
    s2 = np.log(1.0 + (sd * sd) / (mean * mean))
    return np.log(mean) - s2 / 2.0, np.sqrt(s2)


def _apply_errors(rng, tmpl, rm: ReadModel):
    n = tmpl.size
    u = rng.random(n)
    pdel = np.full(n, rm.p_del)
    if rm.homopolymer_del_bias != 1.0 and n > 4:
        # run lengths of homopolymers
        change = np.empty(n, dtype=bool)
        change[0] = True
        change[1:] = tmpl[1:] != tmpl[:-1]
        run_id = np.cumsum(change) - 1
        run_len = np.bincount(run_id)
        inrun = run_len[run_id] >= 4
        pdel = np.where(inrun, np.minimum(rm.p_del * rm.homopolymer_del_bias, 0.5), pdel)
    is_del = u < pdel
    is_sub = (~is_del) & (u < pdel + rm.p_sub)
    out = tmpl.copy()
    ns = int(is_sub.sum())
    if ns:
        out[is_sub] = (out[is_sub] + rng.integers(1, 4, ns, dtype=np.uint8)) & 3
    # insertions: a geometric number of random bases before each template base
    nins = rng.geometric(1.0 - rm.p_ins, n) - 1 if rm.p_ins > 0 else np.zeros(n, dtype=np.int64)
    keep = ~is_del
    counts = nins + keep.astype(np.int64)
    total = int(counts.sum())
    res = rng.integers(0, 4, total, dtype=np.uint8)  # inserted bases are random
    # the kept template base sits at the end of its slot
    ends = np.cumsum(counts) - 1
    res[ends[keep]] = out[keep]
    return res


def make_reads(haps, rm: ReadModel, rng: np.random.Generator, max_bases: int = 0):
    """Returns a list of uint8 reads (0..3); max_bases > 0 stops once the reads hold that
    many bases (the same reads, in the same order, as the start of the full set)."""
    glen = haps[0].size
    mu, sigma = _lognormal_params(rm.mean_len, rm.sd_len)
    reads = []
    target = rm.coverage * glen
    total = 0
    nbases = 0
    while total < target and (max_bases <= 0 or nbases < max_bases):
        L = int(np.clip(np.round(rng.lognormal(mu, sigma)), rm.min_len, min(rm.max_len, glen)))
        h = haps[int(rng.integers(0, len(haps)))]
        L = min(L, h.size)
        s = int(rng.integers(0, h.size - L + 1))
        t = h[s:s + L]
        if rng.random() < 0.5:
            t = (3 - t[::-1]).astype(np.uint8)
        r = _apply_errors(rng, t, rm)
        if r.size < rm.min_len // 2:
            continue
        reads.append(r)
        total += L
        nbases += r.size
    return reads


PACBIO = dict(p_ins=0.09, p_del=0.045, p_sub=0.015)

WORKLOADS = {
    # plain daligner, CPU-runnable: 1 Mbp genome, 20x, mean 8 kbp
    "cfg1": Workload("cfg1", GenomeModel(1_000_000),
                     ReadModel(20, 8000, 4000, 1000, 30000, **PACBIO), seed=1),
    # bacterial scale with repeats: 4.6 Mbp + 40x5 kbp @1.5% + 3x6 kbp @0.2%, 25x, mean 10 kbp
    "cfg2": Workload("cfg2", GenomeModel(4_600_000, repeats=((40, 5000, 0.015), (3, 6000, 0.002))),
                     ReadModel(25, 10000, 5000, 1000, 60000, **PACBIO), seed=2),
    # nanopore-like uneven lengths: 10 Mbp, 30x, mean 20 kbp sd 15 kbp, 1-150 kbp
    "cfg3": Workload("cfg3", GenomeModel(10_000_000),
                     ReadModel(30, 20000, 15000, 1000, 150000, p_ins=0.03, p_del=0.05, p_sub=0.02,
                               homopolymer_del_bias=3.0), seed=3),
    # learned-triage evaluation: 20 Mbp with 10 % interspersed repeat families of 1-8 kbp at
    # 5-15 % divergence, 30x PacBio-like reads, blocks of 200 Mbp (3 blocks)
    "cfg4": Workload("cfg4", GenomeModel(20_000_000, interspersed_frac=0.10, interspersed_len=(1000, 8001),
                                         interspersed_div=(0.05, 0.15)),
                     ReadModel(30, 10000, 5000, 1000, 60000, **PACBIO), seed=4, block_mbp=200),
    # large block pair: 200 Mbp diploid (0.5 % SNPs, 0.05 % short indels between the haplotypes),
    # 35 % interspersed repeat families of 1-10 kbp at 5-15 % divergence, 2 % tandem repeats of
    # period 2-200, 30x PacBio-like reads with mean 15 kbp; blocks of 400 Mbp, the first two
    "cfg5": Workload("cfg5", GenomeModel(200_000_000, interspersed_frac=0.35, interspersed_len=(1000, 10001),
                                         interspersed_div=(0.05, 0.15), tandem_frac=0.02, tandem_period=(2, 201),
                                         diploid_snp=0.005, diploid_indel=0.0005),
                     ReadModel(30, 15000, 7500, 1000, 100000, **PACBIO), seed=5, block_mbp=400, nblocks=2,
                     masks=("dust",)),
    # small cases for tests
    "tiny": Workload("tiny", GenomeModel(60_000),
                     ReadModel(12, 4000, 2000, 1000, 12000, **PACBIO), seed=11),
    "tiny_tandem": Workload("tiny_tandem", GenomeModel(80_000, tandem_frac=0.10, tandem_period=(2, 7)),
                            ReadModel(12, 4000, 2000, 1000, 12000, **PACBIO), seed=13),
    # AT-rich (A, T at 32 %): the frequency weights of daligner -b differ per base
    "tiny_at": Workload("tiny_at", GenomeModel(60_000, base_probs=(0.32, 0.18, 0.18, 0.32)),
                        ReadModel(12, 4000, 2000, 1000, 12000, **PACBIO), seed=15),
    "tiny_at_tandem": Workload("tiny_at_tandem",
                               GenomeModel(80_000, tandem_frac=0.10, tandem_period=(2, 7),
                                           base_probs=(0.32, 0.18, 0.18, 0.32)),
                               ReadModel(12, 4000, 2000, 1000, 12000, **PACBIO), seed=16),
    # strongly skewed (A, T at 40 %) with 20 % tandem repeats: many short weighted windows and
    # many unmasked segments
    "tiny_skew_tandem": Workload("tiny_skew_tandem",
                                 GenomeModel(80_000, tandem_frac=0.20, tandem_period=(2, 7),
                                             base_probs=(0.40, 0.10, 0.10, 0.40)),
                                 ReadModel(12, 4000, 2000, 1000, 12000, **PACBIO), seed=17),
    "small": Workload("small", GenomeModel(200_000, repeats=((6, 3000, 0.015),)),
                      ReadModel(15, 6000, 3000, 1000, 20000, **PACBIO), seed=12),
    # reads of 30-150 kbp: a-positions beyond the 50,000-bp panels of the seed scan
    "long": Workload("long", GenomeModel(250_000, repeats=((4, 3000, 0.01),)),
                     ReadModel(6, 70000, 20000, 30000, 150000, p_ins=0.03, p_del=0.05, p_sub=0.02), seed=14),
}


def generate(w: Workload | str, scale: float = 1.0):
    """Generate (reads, haplotypes) for a workload; scale shrinks the genome for quick runs."""
    if isinstance(w, str):
        w = WORKLOADS[w]
    rng = np.random.Generator(np.random.PCG64(w.seed))
    gm = w.genome
    if scale != 1.0:
        gm = dataclasses.replace(gm, length=max(20000, int(gm.length * scale)))
    haps = make_genome(gm, rng)
    max_bases = int(w.nblocks * w.block_mbp * 1e6) if w.nblocks > 0 else 0
    reads = make_reads(haps, w.reads, rng, max_bases)
    return reads, haps


def write_fasta(path, reads, width=0):
    with open(path, "w") as f:
        letters = np.frombuffer(b"ACGT", dtype=np.uint8)
        for i, r in enumerate(reads):
            f.write(f">sim/{i + 1}/0_{r.size}\n")
            f.write(letters[r].tobytes().decode())
            f.write("\n")


def cached_db(workload: str, seed_offset: int = 0, scale: float = 1.0, cache: str | None = None):
    """Writes (once) the DB of a workload -- seed shifted by 1000 * seed_offset, genome, repeat
    counts and block size scaled by scale -- under cache and returns the path of block 1
    (block n is the same path with its last number replaced)."""
    import os
    import tempfile
    from . import dazzdb
    if cache is None:
        cache = os.environ.get("MARVEL_B200_CACHE", os.path.join(tempfile.gettempdir(), "marvel_b200_bench"))
    w = WORKLOADS[workload]
    w = dataclasses.replace(w, seed=w.seed + 1000 * seed_offset)
    if scale != 1.0:
        g = w.genome
        reps = tuple((max(1, int(round(c * scale))), u, d) for c, u, d in g.repeats)
        w = dataclasses.replace(w, genome=dataclasses.replace(g, length=int(g.length * scale), repeats=reps))
    d = os.path.join(cache, f"{workload}_s{w.seed}_x{scale}")
    root = os.path.join(d, "W")
    if not os.path.exists(root + ".db"):
        reads, _ = generate(w)
        tmp = d + f".tmp{os.getpid()}"
        os.makedirs(tmp, exist_ok=True)
        # a single block unless the workload is split (DBsplit -s<block_mbp>)
        dazzdb.write_db(os.path.join(tmp, "W"), reads, w.block_mbp * scale if w.block_mbp else 100000)
        try:
            os.rename(tmp, d)
        except OSError:   # another process finished first
            pass
    return root + ".1"

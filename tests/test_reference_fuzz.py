"""Differential test against the reference daligner itself: seeded random genomes, read
models and option sets beyond the fixed golden cases (k 10-16, w 4-8, h, e .70-.90, l, s
on both sides of the one-byte trace limit, -M down to 1 GB, -I, -A, -t, -b, -mdust with the
reference DBdust track, block pairs; and daligner2 with its -H), each run by the
reference daligner (daligner2) built from source (oracle/_ref, oracle/Makefile) and by the
device path (GPU) or the oracle (CPU) on the same database; every .las file must be
identical.  Skipped where the reference binary is not built."""
import dataclasses
import os
import subprocess

import numpy as np
import pytest

import daligner_run
from marvel_b200 import dazzdb, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "daligner")
REF2 = os.path.join(ROOT, "oracle", "_ref", "daligner2")
DUST = os.path.join(ROOT, "oracle", "_ref", "DBdust")
N_CASES = 40
N_CASES2 = 20  # daligner2 (modimizer seeds)


def _case(i, variant=1):
    """Option set, genome and read model of case i (seeded): daligner's options, or with
    variant 2 daligner2's (its -H instead of -b)."""
    rng = np.random.default_rng(1000 * variant + i)
    k = int(rng.integers(10, 17))
    w = int(rng.integers(4, 9))
    h = int(rng.integers(max(k + 1, 20), 61))
    e = float(rng.choice([0.70, 0.75, 0.80, 0.85, 0.90]))
    l = int(rng.choice([300, 500, 800, 1000, 1500]))
    s = int(rng.choice([25, 50, 100, 125, 126, 200, 255]))
    flags = [f"-M{int(rng.choice([32, 4, 1]))}", f"-k{k}", f"-w{w}", f"-h{h}", f"-e{e:.2f}", f"-l{l}", f"-s{s}"]
    if rng.random() < 0.3:
        flags.append("-I")
    if rng.random() < 0.3:
        flags.append("-A")
    if rng.random() < 0.3:
        flags.append(f"-t{int(rng.integers(10, 40))}")
    if variant == 1 and rng.random() < 0.25:
        flags.append("-b")
    if variant == 2 and rng.random() < 0.3:
        flags.append(f"-H{int(rng.integers(2000, 8000))}")
    if rng.random() < 0.25:
        flags.append("-mdust")
    pair = rng.random() < 0.4
    err = float(rng.uniform(0.04, 0.16))  # total error rate of the reads
    genome = synth.GenomeModel(int(rng.integers(40_000, 90_000)),
                               repeats=((int(rng.integers(0, 6)), int(rng.integers(1000, 4000)),
                                         float(rng.uniform(0.0, 0.03))),))
    reads = synth.ReadModel(int(rng.integers(8, 16)), int(rng.integers(2500, 7000)), 2000, 800, 15000,
                            p_ins=err * 0.6, p_del=err * 0.3, p_sub=err * 0.1)
    wl = synth.Workload(f"fuzz{variant}_{i}", genome, reads, seed=2000 * variant + i)
    return wl, flags, pair


def _reference_run(i, tmp_path, variant=1):
    """Case i's database under tmp_path/db and the reference daligner's (daligner2's) .las
    files there; returns (db dir, flags, blocks)."""
    wl, flags, pair = _case(i, variant)
    reads, _ = synth.generate(wl)
    total = sum(r.size for r in reads)
    d = tmp_path / "db"
    d.mkdir()
    # a block pair: two blocks of about half the bases each
    dazzdb.write_db(str(d / "G"), reads, (total / 2 + 1) / 1e6 if pair else 200)
    blocks = ["G.1", "G.2"] if pair else ["G.1", "G.1"]
    if "-mdust" in flags:
        subprocess.run([DUST, "G"], cwd=str(d), check=True, stdout=subprocess.DEVNULL)
    cmd = [REF, "-j4"] if variant == 1 else [REF2, "-T4", "-Pout"]
    subprocess.run(cmd + flags + blocks, cwd=str(d), check=True, stdout=subprocess.DEVNULL)
    return d, flags, blocks


def _compare(i, impl, tmp_path, variant=1):
    d, flags, blocks = _reference_run(i, tmp_path, variant)
    names = daligner_run.run(str(d), flags, blocks, str(tmp_path / impl), impl, variant=variant)
    assert names
    for n in names:
        assert os.path.exists(d / n), f"case {i} {flags}: the reference wrote no {n}"
        ok, msg = dazzdb.las_equal(str(tmp_path / impl / n), str(d / n))
        assert ok, f"case {i} {flags} {blocks}: {n}: {msg}"


needs_ref = pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(REF2) and os.path.exists(DUST)),
                               reason="the reference daligner is not built (make -C oracle ref)")


@needs_ref
@pytest.mark.parametrize("i", range(N_CASES))
def test_oracle_equals_reference_daligner(i, tmp_path):
    _compare(i, "oracle", tmp_path)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("i", range(N_CASES))
def test_device_path_equals_reference_daligner(i, tmp_path):
    _compare(i, "gpu", tmp_path)


@needs_ref
@pytest.mark.parametrize("i", range(N_CASES2))
def test_oracle_equals_reference_daligner2(i, tmp_path):
    _compare(i, "oracle", tmp_path, variant=2)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("i", range(N_CASES2))
def test_device_path_equals_reference_daligner2(i, tmp_path):
    _compare(i, "gpu", tmp_path, variant=2)


# ---- DBdust: random databases and parameters against the reference DBdust's track

N_DUST = 20


def _dust_case(i):
    rng = np.random.default_rng(5000 + i)
    kw = dict(window=int(rng.choice([16, 32, 48, 64, 100, 128])), thresh=float(rng.choice([1.0, 1.5, 2.0, 2.5, 3.0])),
              mflag=int(rng.choice([5, 8, 10, 15])), biased=bool(rng.random() < 0.3))
    at = float(rng.uniform(0.25, 0.42))  # A and T share of the genome
    genome = synth.GenomeModel(int(rng.integers(30_000, 80_000)), tandem_frac=float(rng.uniform(0.0, 0.25)),
                               tandem_period=(2, int(rng.integers(3, 12))),
                               base_probs=(at, 0.5 - at, 0.5 - at, at))
    reads = synth.ReadModel(6, 4000, 2000, 800, 12000, **synth.PACBIO)
    return synth.Workload(f"dust{i}", genome, reads, seed=6000 + i), kw


def _dust_flags(kw):
    f = [f"-w{kw['window']}", f"-t{kw['thresh']}", f"-m{kw['mflag']}"]
    return f + (["-b"] if kw["biased"] else [])


def _dust_reference(i, tmp_path):
    wl, kw = _dust_case(i)
    reads, _ = synth.generate(wl)
    d = tmp_path / "db"
    d.mkdir()
    dazzdb.write_db(str(d / "G"), reads, 200)
    subprocess.run([DUST] + _dust_flags(kw) + ["G"], cwd=str(d), check=True, stdout=subprocess.DEVNULL)
    a = open(d / ".G.dust.anno", "rb").read()
    anno = np.frombuffer(a[8:], "<i8")
    data = np.fromfile(str(d / ".G.dust.data"), "<i4")
    return dazzdb.open_block(str(d / "G.1")), kw, anno, data


@needs_ref
@pytest.mark.parametrize("i", range(N_DUST))
def test_oracle_dust_equals_reference_dbdust(i, tmp_path):
    import oracle
    blk, kw, anno, data = _dust_reference(i, tmp_path)
    oa, od = oracle.dust(blk, **kw)
    assert np.array_equal(oa, anno) and np.array_equal(od, data), kw


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("i", range(N_DUST))
def test_device_dust_equals_reference_dbdust(i, tmp_path):
    import marvel_b200 as mb
    blk, kw, anno, data = _dust_reference(i, tmp_path)
    ctx = mb.Context()
    ctx.load_block(0, blk)
    ga, gd = ctx.dust(0, blk.freq, **kw)
    ctx.close()
    assert np.array_equal(ga, anno) and np.array_equal(gd, data), kw


# ---- LAsort: the records of a random case's .las files, shuffled, against the reference LAsort

LASORT = os.path.join(ROOT, "oracle", "_ref", "LAsort")
N_LASORT = 10


def _raw_records(path):
    """(trace spacing, the byte string of each record: 40-byte header with its pad + trace)."""
    data = open(path, "rb").read()
    n = int(np.frombuffer(data[:8], "<i8")[0])
    ts = int(np.frombuffer(data[8:12], "<i4")[0])
    tb = 1 if ts <= 125 else 2
    out, o = [], 12
    for _ in range(n):
        tlen = int(np.frombuffer(data[o:o + 4], "<i4")[0])
        out.append(data[o:o + 40 + tlen * tb])
        o += 40 + tlen * tb
    return ts, out


def _lasort_reference(i, tmp_path):
    d, flags, blocks = _reference_run(i, tmp_path)
    recs, ts = [], None
    for root, _, files in os.walk(d):
        for f in sorted(files):
            if f.endswith(".las"):
                ts, r = _raw_records(os.path.join(root, f))
                recs += r
    rng = np.random.default_rng(7000 + i)
    recs = [recs[j] for j in rng.permutation(len(recs))]
    src = tmp_path / "in.las"
    with open(src, "wb") as f:
        f.write(np.int64(len(recs)).tobytes())
        f.write(np.int32(ts).tobytes())
        for r in recs:
            f.write(r)
    subprocess.run([LASORT, "in.las"], cwd=str(tmp_path), check=True, stdout=subprocess.DEVNULL)
    return src, tmp_path / "in.S.las"


needs_lasort = pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(LASORT)),
                                  reason="the reference LAsort is not built (make -C oracle ref)")


@needs_lasort
@pytest.mark.parametrize("i", range(N_LASORT))
def test_oracle_las_sort_equals_reference_lasort(i, tmp_path):
    import las_sort
    src, want = _lasort_reference(i, tmp_path)
    las_sort.las_sort(str(src), str(tmp_path / "o.las"))
    ok, msg = dazzdb.las_equal(str(tmp_path / "o.las"), str(want), key="lasort", pad=True)
    assert ok, msg


@pytest.mark.gpu
@needs_lasort
@pytest.mark.parametrize("i", range(N_LASORT))
def test_device_las_sort_equals_reference_lasort(i, tmp_path):
    import marvel_b200 as mb
    src, want = _lasort_reference(i, tmp_path)
    ctx = mb.Context()
    ctx.las_sort(str(src), str(tmp_path / "g.las"))
    ctx.close()
    ok, msg = dazzdb.las_equal(str(tmp_path / "g.las"), str(want), key="lasort", pad=True)
    assert ok, msg


# ---- LAmerge: the per-block .las directories of a random multi-block run

LAMERGE = os.path.join(ROOT, "oracle", "_ref", "LAmerge")
N_LAMERGE = 6


def _lamerge_reference(i, tmp_path):
    wl, flags, _ = _case(100 + i)
    flags = [f for f in flags if f != "-mdust"]
    reads, _ = synth.generate(wl)
    total = sum(r.size for r in reads)
    d = tmp_path / "db"
    d.mkdir()
    dazzdb.write_db(str(d / "G"), reads, (total / 3 + 1) / 1e6)
    nb = len(dazzdb.read_stub(str(d / "G.db"))[3]) - 1  # the blocks DBsplit's rule gave
    for b in range(1, nb + 1):  # HPCdaligner's jobs: block b against itself and the blocks before it
        subprocess.run([REF, "-r1", "-j4"] + flags + [f"G.{b}"] + [f"G.{c}" for c in range(b, 0, -1)], cwd=str(d),
                       check=True, stdout=subprocess.DEVNULL)
    for b in range(1, nb + 1):
        subprocess.run([LAMERGE, "-n", "8", "G.db", f"G.{b}.las", "%03d_%05d" % (1, b)], cwd=str(d), check=True,
                       stdout=subprocess.DEVNULL)
    return d, nb


needs_lamerge = pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(LAMERGE)),
                                   reason="the reference LAmerge is not built (make -C oracle ref)")


@pytest.mark.gpu
@needs_lamerge
@pytest.mark.parametrize("i", range(N_LAMERGE))
def test_device_las_merge_equals_reference_lamerge(i, tmp_path):
    from marvel_b200 import lamerge
    d, nb = _lamerge_reference(i, tmp_path)
    for b in range(1, nb + 1):
        out = tmp_path / f"G.{b}.las"
        assert lamerge.main(["-n", "8", str(d / "G.db"), str(out), str(d / ("%03d_%05d" % (1, b)))]) == 0
        ok, msg = dazzdb.las_equal(str(out), str(d / f"G.{b}.las"), key="overlap", pad=True)
        assert ok, f"case {i} block {b}: {msg}"


# ---- the reference's own driver linked against the library (the link-time drop-in)

RELINKED = os.path.join(ROOT, "oracle", "_ref", "daligner_relinked")
N_RELINK = 10


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(RELINKED)),
                    reason="oracle/_ref/daligner_relinked is not built (make -C oracle ref)")
@pytest.mark.parametrize("i", range(N_RELINK))
def test_relinked_reference_driver_equals_reference_daligner(i, tmp_path):
    """dalign/daligner.c, unmodified, linked against libgpudalign.so in place of the
    reference's filter.c and align.c: the same .las files as the reference daligner."""
    import shutil
    d, flags, blocks = _reference_run(200 + i, tmp_path)
    g = tmp_path / "relinked"
    g.mkdir()
    for f in os.listdir(d):
        if os.path.isfile(d / f):
            shutil.copy(d / f, g / f)
    r = subprocess.run([RELINKED, "-j4"] + flags + blocks, cwd=str(g), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names = [os.path.relpath(os.path.join(root, f), d) for root, _, fs in os.walk(d) for f in fs if f.endswith(".las")]
    assert names
    for n in names:
        ok, msg = dazzdb.las_equal(str(g / n), str(d / n))
        assert ok, f"case {200 + i} {flags} {blocks}: {n}: {msg}"


# ---- the daligner command line of this package on the same random cases

CLI = os.path.join(ROOT, "marvel_b200", "daligner_gpu")
N_CLI = 10


@pytest.mark.gpu
@pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(CLI)),
                    reason="the reference daligner or marvel_b200/daligner_gpu is not built")
@pytest.mark.parametrize("i", range(N_CLI))
def test_command_line_equals_reference_daligner(i, tmp_path):
    """marvel_b200/daligner_gpu, given the reference's command line, writes the reference
    daligner's .las files (option parsing, mask tracks, file names and the two-file split)."""
    import shutil
    d, flags, blocks = _reference_run(300 + i, tmp_path)
    g = tmp_path / "cli"
    g.mkdir()
    for f in os.listdir(d):
        if os.path.isfile(d / f):
            shutil.copy(d / f, g / f)
    r = subprocess.run([CLI, "-j4"] + flags + blocks, cwd=str(g), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names = [os.path.relpath(os.path.join(root, f), d) for root, _, fs in os.walk(d) for f in fs if f.endswith(".las")]
    assert names
    for n in names:
        ok, msg = dazzdb.las_equal(str(g / n), str(d / n))
        assert ok, f"case {300 + i} {flags} {blocks}: {n}: {msg}"

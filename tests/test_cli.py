"""The daligner command line over the GPU path (marvel_b200/daligner_gpu)."""
import glob
import os
import shutil
import subprocess

import pytest

from golden_cases import cases, d2_cases, load
from marvel_b200 import dazzdb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "marvel_b200", "daligner_gpu")
CLI2 = os.path.join(ROOT, "marvel_b200", "daligner2_gpu")


def _run(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True)


def _copy_db(src, dst):
    for f in glob.glob(os.path.join(src, "*")) + glob.glob(os.path.join(src, ".*")):
        if os.path.isfile(f):
            shutil.copy(f, dst)


@pytest.mark.parametrize("args,msg", [
    (["-j3", "G.1", "G.1"], "Must be a power of 2"),
    (["-e.4", "G.1", "G.1"], "Average correlation must be in [.5,1.)"),
    (["-Dhost:1", "G.1", "G.1"], "-D (dynamic mask server) is not supported"),
    (["-x", "G.1", "G.1"], "Unsupported option"),
    (["G.1"], "at least one target and one subject block are required"),
])
def test_cli_rejects_bad_arguments(args, msg, tmp_path):
    r = _run(args, str(tmp_path))
    assert r.returncode == 1
    assert msg in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", cases())
def test_cli_matches_reference_golden(name, tmp_path):
    d, meta = load(name)
    _copy_db(d, str(tmp_path))
    r = _run(["-j4"] + meta["flags"] + meta["blocks"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    for n in meta["las"]:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["self_s200_t20", "pair_blocks", "self_asym_lowmem", "pair_dust_biased"])
def test_cli_verbose_report_matches_reference(name, tmp_path):
    """-v prints the reference's report (index sizes, pair cap, hit counts, seed and
    confirmed hits) character for character (tests/golden/make_verbose_golden.py)."""
    d, meta = load(name)
    _copy_db(d, str(tmp_path))
    r = _run(["-v", "-j4"] + meta["flags"] + meta["blocks"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    with open(os.path.join(d, "verbose.txt")) as f:
        assert r.stdout == f.read()


@pytest.mark.parametrize("args,msg", [
    (["-x", "G.1", "G.1"], "-x is an illegal option"),
    (["-e.5", "G.1", "G.1"], "Average correlation must be in [.7,1.)"),
    (["-k40", "G.1", "G.1"], "K-mer length must be 32 or less"),
    (["-kx", "G.1", "G.1"], "-k argument is not an integer"),
    (["-T0", "G.1", "G.1"], "Number of threads must be positive"),
    (["G.1"], "Usage: daligner"),
])
def test_cli2_rejects_bad_arguments(args, msg, tmp_path):
    r = subprocess.run([CLI2] + args, cwd=str(tmp_path), capture_output=True, text=True)
    assert r.returncode == 1
    assert msg in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", d2_cases())
def test_cli2_matches_reference_daligner2_golden(name, tmp_path):
    d, meta = load(name)
    _copy_db(d, str(tmp_path))
    blocks = meta["blocks"]
    if blocks[0] != blocks[1]:
        blocks = [blocks[0], blocks[1].rpartition(".")[2]]   # a bare number: a block of the same DB
    r = subprocess.run([CLI2, "-T4", "-Pout"] + meta["flags"] + blocks, cwd=str(tmp_path), capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    for n in meta["las"]:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"
    # -S: the valid files stay as they are
    stamp = {n: os.stat(tmp_path / n).st_mtime_ns for n in meta["las"]}
    r = subprocess.run([CLI2, "-S", "-T4", "-Pout"] + meta["flags"] + blocks, cwd=str(tmp_path), capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    assert all(os.stat(tmp_path / n).st_mtime_ns == t for n, t in stamp.items())

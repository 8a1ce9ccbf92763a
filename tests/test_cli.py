"""The daligner command line over the GPU path (marvel_b200/daligner_gpu)."""
import glob
import os
import shutil
import subprocess

import pytest

from golden_cases import cases, load
from marvel_b200 import dazzdb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "marvel_b200", "daligner_gpu")


def _run(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True)


def _copy_db(src, dst):
    for f in glob.glob(os.path.join(src, "*")) + glob.glob(os.path.join(src, ".*")):
        if os.path.isfile(f):
            shutil.copy(f, dst)


@pytest.mark.parametrize("args,msg", [
    (["-j3", "G.1", "G.1"], "Must be a power of 2"),
    (["-e.4", "G.1", "G.1"], "Average correlation must be in [.5,1.)"),
    (["-b", "G.1", "G.1"], "-b (biased k-mer sampling) is not supported"),
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

"""Failure paths, made to happen without faulting anything.

* Capacity overflow (GPU): the aligner starts with tiny pebble, trace, path and output
  capacities (test hook gd_set_capacities); every overflow is detected on the device,
  reported through the status word, grown on the host and the alignment stage re-run.  The
  output must equal the reference's golden files, with re-runs counted.
* Wait expiry (GPU): the radix sort's bounded mbarrier wait runs out on an mbarrier armed
  for a copy that is never issued (test hook gd_test_wait_expiry, nothing in flight); the
  sort's check reports it once and clears it, and the next sort is bit-exact.
* Malformed input (CPU): a truncated .idx or .bps and malformed track files make the
  daligner command line exit with status 1 and a message, as the reference's EXIT does
  (db/DB.h:36), before any device work.
"""
import glob
import os
import shutil
import subprocess

import numpy as np
import pytest

import daligner_run
from golden_cases import load
from marvel_b200 import dazzdb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "marvel_b200", "daligner_gpu")


def _copy_db(src, dst):
    for f in glob.glob(os.path.join(src, "*")) + glob.glob(os.path.join(src, ".*")):
        if os.path.isfile(f):
            shutil.copy(f, dst)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["self_default", "pair_blocks", "self_s200_t20", "self_long_panels"])
def test_capacity_overflow_regrows_and_reruns_with_identical_output(name, tmp_path):
    d, meta = load(name)
    st = {}
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu",
                             ctx_hook=lambda ctx: ctx.set_capacities(pebbles=64, traces=64, paths=2, records=16,
                                                                     trace_bytes=256),
                             stats_out=st)
    assert sum(st["reruns"]) > 0, "the tiny capacities should have forced re-runs"
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.gpu
def test_sort_wait_expiry_is_reported_once_and_cleared(tmp_path):
    import marvel_b200 as mb
    ctx = mb.Context()
    rc, msg = ctx.test_wait_expiry(2000)
    assert rc == -1 and "wait limit" in msg, (rc, msg)
    ctx.close()
    # the flag was cleared by the check: the next block comparison sorts and checks normally
    d, meta = load("self_default")
    names = daligner_run.run(d, meta["flags"], meta["blocks"], str(tmp_path), "gpu")
    for n in names:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, msg


def _cli(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True)


def _truncate(path, size):
    with open(path, "r+b") as f:
        f.truncate(size)


def test_truncated_idx_exits_1(tmp_path):
    d, meta = load("self_default")
    _copy_db(d, str(tmp_path))
    _truncate(str(tmp_path / ".G.idx"), 88 + 32 * 3)
    r = _cli(["-M32", "G.1", "G.1"], str(tmp_path))
    assert r.returncode == 1 and "Index file (.idx) of G is junk" in r.stderr, r.stderr


def test_truncated_bps_exits_1(tmp_path):
    d, meta = load("self_default")
    _copy_db(d, str(tmp_path))
    p = str(tmp_path / ".G.bps")
    _truncate(p, os.path.getsize(p) // 2)
    r = _cli(["-M32", "G.1", "G.1"], str(tmp_path))
    assert r.returncode == 1 and "Read of .bps file failed" in r.stderr, r.stderr


def _dust_case(tmp_path):
    d, meta = load("pair_dust")
    _copy_db(d, str(tmp_path))
    return [f for f in meta["flags"] if not f.startswith("-M")]


def test_track_anno_with_bad_record_size_exits_1(tmp_path):
    flags = _dust_case(tmp_path)
    p = str(tmp_path / ".G.dust.anno")
    a = np.fromfile(p, np.uint8)
    a[4:8] = np.frombuffer(np.int32(3).tobytes(), np.uint8)   # record size 3: neither 4 nor 8
    a.tofile(p)
    r = _cli(["-M32"] + flags + ["G.1", "G.2"], str(tmp_path))
    assert r.returncode == 1 and "Unable to load track dust" in r.stdout, (r.stdout, r.stderr)
    assert "annotation file is junk" in r.stderr


def test_track_anno_out_of_order_exits_1(tmp_path):
    flags = _dust_case(tmp_path)
    p = str(tmp_path / ".G.dust.anno")
    raw = np.fromfile(p, np.uint8)
    size = int(raw[4:8].view(np.int32)[0])
    anno = raw[8:].view(np.int64 if size == 8 else np.int32).copy()
    i = int(np.argmax(anno[1:] > anno[:-1])) + 1          # a read with intervals: make its end precede its start
    anno[i] = anno[i - 1] - 8
    raw[8:] = anno.view(np.uint8)
    raw.tofile(p)
    r = _cli(["-M32"] + flags + ["G.1", "G.2"], str(tmp_path))
    assert r.returncode == 1 and "Unable to load track dust" in r.stdout, (r.stdout, r.stderr)
    assert "data file is junk" in r.stderr


def test_truncated_track_data_exits_1(tmp_path):
    flags = _dust_case(tmp_path)
    p = str(tmp_path / ".G.dust.data")
    _truncate(p, 8)
    r = _cli(["-M32"] + flags + ["G.1", "G.2"], str(tmp_path))
    assert r.returncode == 1 and "Unable to load track dust" in r.stdout, (r.stdout, r.stderr)
    assert "data file is junk" in r.stderr

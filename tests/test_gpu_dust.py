"""DBdust on the device (gd_dust) against the reference DBdust's tracks and the CPU
restatement: identical interval tracks, byte for byte."""
import os
import shutil

import numpy as np
import pytest

from dust_cases import GOLD, read_track, runs
from marvel_b200 import dazzdb, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mb():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200
    return marvel_b200


@pytest.mark.parametrize("track,db,kw", runs())
def test_gpu_dust_matches_reference(mb, track, db, kw):
    blk = dazzdb.open_block(os.path.join(GOLD, db))
    ctx = mb.Context()
    ctx.load_block(0, blk)
    anno, data = ctx.dust(0, blk.freq, **kw)
    ctx.close()
    n, ra, rd = read_track(os.path.join(GOLD, f".{db}.{track}"))
    assert np.array_equal(anno, ra) and np.array_equal(data, rd)


def test_gpu_dust_cli_writes_the_reference_files(mb, tmp_path):
    from marvel_b200 import dbdust
    for f in ("G.db", ".G.idx", ".G.bps"):
        shutil.copy(os.path.join(GOLD, f), tmp_path / f)
    assert dbdust.main([str(tmp_path / "G")]) == 0
    assert dbdust.main([str(tmp_path / "G.2")]) == 0
    for base in (".G.dust", ".G.2.dust"):
        for ext in ("anno", "data"):
            assert open(tmp_path / f"{base}.{ext}", "rb").read() == open(os.path.join(GOLD, f"{base}.{ext}"),
                                                                          "rb").read()


@pytest.mark.parametrize("biased", [False, True])
def test_gpu_dust_matches_oracle_on_cfg1(mb, tmp_path, biased):
    """The 1 Mbp / 20x workload (2.5 k reads, 21 Mbp) against the CPU restatement."""
    import oracle
    reads, _ = synth.generate("cfg1")
    dazzdb.write_db(str(tmp_path / "C"), reads, 200)
    blk = dazzdb.open_block(str(tmp_path / "C.1"))
    ctx = mb.Context()
    ctx.load_block(0, blk)
    anno, data = ctx.dust(0, blk.freq, biased=biased)
    ctx.close()
    oa, od = oracle.dust(blk, biased=biased)
    assert np.array_equal(anno, oa) and np.array_equal(data, od)

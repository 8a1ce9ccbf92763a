"""DBdust's CPU restatement (oracle/dust_oracle.c) against the reference DBdust's tracks."""
import os

import numpy as np
import pytest

from dust_cases import GOLD, read_track, runs
from marvel_b200 import dazzdb


@pytest.mark.parametrize("track,db,kw", runs())
def test_oracle_dust_matches_reference(track, db, kw):
    import oracle
    blk = dazzdb.open_block(os.path.join(GOLD, db))
    anno, data = oracle.dust(blk, **kw)
    n, ra, rd = read_track(os.path.join(GOLD, f".{db}.{track}"))
    assert n == blk.nreads
    assert np.array_equal(anno, ra) and np.array_equal(data, rd)
    assert rd.size > 100

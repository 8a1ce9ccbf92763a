"""LAmerge's CPU restatement (oracle/las_sort.py) against the reference LAmerge's merged
files of the 3-block plan (tests/golden/hpc_3blocks), pad words included, tied keys in any
order."""
import json
import os

import pytest

from marvel_b200 import dazzdb

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hpc_3blocks")


def merge_cases():
    meta = json.load(open(os.path.join(GOLD, "hpc.json")))
    return list(zip(meta["merged"], meta["merge_dirs"]))


@pytest.mark.parametrize("merged,src", merge_cases())
def test_oracle_las_merge_matches_reference(merged, src, tmp_path):
    import las_sort
    d = os.path.join(GOLD, src)
    files = sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(".las"))
    assert len(files) == 3
    las_sort.las_merge(files, str(tmp_path / "m.las"))
    ok, msg = dazzdb.las_equal(str(tmp_path / "m.las"), os.path.join(GOLD, merged), key="overlap", pad=True)
    assert ok, msg

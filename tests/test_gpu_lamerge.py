"""LAmerge on the device (gd_las_merge, `python -m marvel_b200.lamerge`) against the
reference LAmerge's merged files of the 3-block plan: same records and bytes (pad words
included), tied keys in any order."""
import json
import os

import pytest

from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hpc_3blocks")


def test_gpu_lamerge_matches_reference(tmp_path):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from marvel_b200 import lamerge
    meta = json.load(open(os.path.join(GOLD, "hpc.json")))
    for merged, src in zip(meta["merged"], meta["merge_dirs"]):
        out = tmp_path / merged
        assert lamerge.main(["-n", "8", os.path.join(GOLD, "G.db"), str(out), os.path.join(GOLD, src)]) == 0
        ok, msg = dazzdb.las_equal(str(out), os.path.join(GOLD, merged), key="overlap", pad=True)
        assert ok, f"{merged}: {msg}"

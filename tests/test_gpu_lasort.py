"""LAsort on the device (gd_las_sort) against the reference LAsort's outputs and the CPU
restatement: same records, same bytes (pad words included), tied keys in any order."""
import os

import pytest

from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lasort")


@pytest.mark.parametrize("name", ["cat", "s200"])
def test_gpu_las_sort_matches_reference(name, tmp_path):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200 as mb
    import las_sort
    ctx = mb.Context()
    n = ctx.las_sort(os.path.join(GOLD, name + ".las"), str(tmp_path / "g.las"))
    n2 = ctx.las_sort(str(tmp_path / "g.las"), str(tmp_path / "g2.las"))   # idempotent
    ctx.close()
    ok, msg = dazzdb.las_equal(str(tmp_path / "g.las"), os.path.join(GOLD, name + ".S.las"), key="lasort", pad=True)
    assert ok, msg
    assert n == n2 and open(tmp_path / "g.las", "rb").read() == open(tmp_path / "g2.las", "rb").read()
    las_sort.las_sort(os.path.join(GOLD, name + ".las"), str(tmp_path / "o.las"))
    ok, msg = dazzdb.las_equal(str(tmp_path / "g.las"), str(tmp_path / "o.las"), key="lasort", pad=True)
    assert ok, msg


def test_gpu_las_sort_cli_and_empty_file(tmp_path):
    import shutil
    import numpy as np
    from marvel_b200 import lasort
    shutil.copy(os.path.join(GOLD, "cat.las"), tmp_path / "U.las")
    with open(tmp_path / "E.las", "wb") as f:
        f.write(np.int64(0).tobytes() + np.int32(100).tobytes())
    assert lasort.main([str(tmp_path / "U"), str(tmp_path / "E.las")]) == 0
    ok, msg = dazzdb.las_equal(str(tmp_path / "U.S.las"), os.path.join(GOLD, "cat.S.las"), key="lasort", pad=True)
    assert ok, msg
    assert dazzdb.read_las(str(tmp_path / "E.S.las"))[1].size == 0

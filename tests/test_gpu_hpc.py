"""The multi-block driver on the GPU: HPCdaligner's default plan for a 3-block DB, run
through daligner_gpu, writes the same nine .las files as the reference daligner running the
reference's plan (tests/golden/hpc_3blocks), and the plan's merge step writes the reference
LAmerge's three merged files."""
import json
import os
import shutil

import pytest

from marvel_b200 import dazzdb, hpc

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hpc_3blocks")


def test_three_block_plan_matches_reference(tmp_path):
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    meta = json.load(open(os.path.join(GOLD, "hpc.json")))
    for f in ("G.db", ".G.idx", ".G.bps"):
        shutil.copy(os.path.join(GOLD, f), tmp_path / f)
    o = hpc.HpcOptions()
    db = str(tmp_path / "G")
    assert hpc.plan_text(db, 1, 3, o).splitlines()[1:4] == [
        ln.replace("G.", str(tmp_path) + "G.") for ln in meta["plan"].splitlines()[1:4]]
    calls, secs = hpc.run(db, o, merge=True)
    assert calls == 3
    for m in meta["merged"]:   # the plan's LAmerge step, merged on the GPU
        ok, msg = dazzdb.las_equal(str(tmp_path / m), os.path.join(GOLD, m), key="overlap", pad=True)
        assert ok, f"{m}: {msg}"
        os.remove(tmp_path / m)
    got = sorted(os.path.relpath(os.path.join(r, f), tmp_path) for r, _, fs in os.walk(tmp_path) for f in fs
                 if f.endswith(".las"))
    assert got == meta["las"]
    for n in got:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(GOLD, n))
        assert ok, f"{n}: {msg}"

"""The aligner schedule autotuner: its candidate schedules (host logic, CPU) and one tuning
pass on a golden case (GPU), where every candidate must give the same records."""
import os

import numpy as np
import pytest

from marvel_b200 import autotune, dazzdb


def test_candidates_cover_every_instance_with_one_kind_per_class():
    edges = [8000, 20000, 60000]
    cands = autotune.candidates(edges)
    names = [c[0] for c in cands]
    assert len(set(names)) == len(names)
    seen = set()
    for name, e, kinds in cands:
        assert len(kinds) == len(e) + 1, name
        assert set(kinds) <= {0, 1, 2}, name
        seen.update(kinds)
    assert seen == {0, 1, 2}
    # the persistent launches hold one instance for the one class
    assert ("persistent, duo instance", [], [2]) in cands


def test_length_edges_are_increasing_and_inside_the_pair_lengths():
    rng = np.random.default_rng(3)

    class B:
        rlen = rng.integers(1000, 30000, 2000)

    e = autotune.length_edges(B, None, 4)
    assert e == sorted(e) and len(e) <= 3
    assert all(2000 <= x <= 60000 for x in e)


@pytest.mark.gpu
def test_tuning_a_golden_case_keeps_its_records():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import marvel_b200 as mb
    from golden_cases import load
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    ctx = mb.Context()
    ctx.set_filter_params(14, 6, 0, 35)
    ctx.new_align_spec(0.70, 100, A.freq)
    ctx.set_globals(2000, False, 32 << 30)
    ctx.load_block(0, A)
    rep = autotune.tune(ctx, A, None, nclasses=3, repeats=1)  # raises if two schedules differ
    assert rep["chosen"] in {c["schedule"] for c in rep["candidates"]}
    assert len(rep["candidates"]) == len(autotune.candidates(autotune.length_edges(A, None, 3)))
    ctx.close()

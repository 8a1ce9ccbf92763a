"""The multi-block driver's host side (no GPU): HPCdaligner's plan against the reference's
printed plans (tests/golden/hpc_plans.json), the split of a plan over ranks, and a 2-rank
gloo run of the sharded driver with a stand-in for the GPU calls."""
import json
import os
import socket

import pytest

from marvel_b200 import dazzdb, hpc, synth

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hpc_plans.json")


@pytest.fixture(scope="module")
def db4(tmp_path_factory):
    d = tmp_path_factory.mktemp("hpc")
    reads, _ = synth.generate("tiny")
    os.makedirs(d / "sub")
    dazzdb.write_db(str(d / "G"), reads, 0.2)
    dazzdb.write_db(str(d / "sub" / "G"), reads, 0.2)
    assert hpc.db_blocks(str(d / "G")) == 4
    return d


def test_plans_match_reference(db4, monkeypatch):
    monkeypatch.chdir(db4)
    gold = json.load(open(GOLD))
    assert len(gold["plans"]) >= 10
    for case in gold["plans"]:
        db, fb, lb, o, _ = hpc.parse_args(case["args"].split())
        assert hpc.plan_text(db, fb, lb, o) == case["plan"], case["args"]


def test_plan_covers_every_block_pair_once():
    for consecutive in (False, True):
        for n in (1, 2, 5, 9):
            for dal, dd in ((4, 0), (1, 1), (3, 2)):
                o = hpc.HpcOptions(dal=dal, dal_diag=dd, consecutive=consecutive)
                pairs = [(a, b) for a, bl in hpc.plan(1, n, o) for b in bl]
                want = {(a, b) for a in range(1, n + 1) for b in range(1, n + 1)
                        if (b >= a if consecutive else b <= a)}
                assert sorted(pairs) == sorted(want)
                assert all(len(bl) <= max(dal, dd or dal) for _, bl in hpc.plan(1, n, o))


def test_assign_partitions_the_plan():
    jobs = hpc.plan(1, 12, hpc.HpcOptions(dal=3))
    for world in (1, 2, 3, 4, 8):
        parts = [hpc.assign(jobs, world, r) for r in range(world)]
        flat = [j for p in parts for j in p]
        assert sorted(flat) == sorted(jobs)
        loads = [sum(len(bl) for _, bl in p) for p in parts]
        assert max(loads) - min(loads) <= max(len(bl) for _, bl in jobs)


def test_exec_flags_pass_the_memory_limit_as_M():
    o = hpc.HpcOptions(M=8, s=50, no_trace=True, k=16)
    assert "-s8" in hpc.daligner_flags(o, False)          # the reference's plan text
    f = hpc.exec_flags(o)
    assert "-M8" in f and "-s50" in f and "-s8" not in f and not any(x.startswith("-j") for x in f)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, db, out):
    import time
    import torch.distributed as dist
    from marvel_b200 import hpc as h
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ran = []

    def fake(cwd, args):   # stands in for one daligner_gpu call
        ran.append(args)
        time.sleep(0.01 * (1 + rank))

    merged = []
    calls, secs = h.run(db, h.HpcOptions(dal=2), executor=fake, merge=True,
                        merger=lambda src, out: merged.append(os.path.basename(out)))
    with open(os.path.join(out, f"rank{rank}.json"), "w") as f:
        json.dump({"ran": ran, "calls": calls, "secs": secs, "merged": merged}, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_the_plan_over_gloo(db4, tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(db4 / "G"), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    jobs = hpc.plan(1, 4, hpc.HpcOptions(dal=2))
    ran = [tuple(a) for r in res for a in r["ran"]]
    want = [tuple(hpc.exec_flags(hpc.HpcOptions(dal=2)) + [f"G.{a}"] + [f"G.{b}" for b in bl]) for a, bl in jobs]
    assert sorted(ran) == sorted(want)                        # every call exactly once
    assert res[0]["ran"] and res[1]["ran"]                    # both ranks worked
    assert res[0]["calls"] == res[1]["calls"] == len(jobs)    # sum over ranks
    assert res[0]["secs"] == res[1]["secs"] > 0               # max over ranks, same on all
    assert sorted(res[0]["merged"] + res[1]["merged"]) == [f"G.{i}.las" for i in range(1, 5)]

"""Multi-block, multi-GPU driver: HPCdaligner's job plan, run as one process per GPU.

HPCdaligner (dalign/HPCdaligner.c) writes a plan of `daligner` calls that together compare
every block of a DB with every other (block i against blocks j <= i; each call compares one
A block with up to --dal B blocks) and the LAmerge calls that follow.  The block pairs are
independent, so the GPU build shards the plan's calls over the ranks of one node -- one
process per GPU, no collective on the data path -- and runs each call through the sm_100a
command-line driver (`daligner_gpu`, the same options and .las files as daligner), which
builds the A block's k-mer index once and reuses it for every B block of the call
(dalign/daligner.c:945-958).  The only collective is the final reduction of the per-rank
statistics (max of the wall time, sum of the calls run).

`plan()` restates the job enumeration of HPCdaligner.c:573-790 (both orders: the default
diagonal-first rounds and -X's row order); `plan_text()` restates its printed plan,
including its quirks (a memory limit is printed as a second `-s`, and a DB path with a
directory loses the `/` between the directory and the DB name) so that it can be compared
with the reference's output byte for byte.
"""
from __future__ import annotations

import math
import os
import subprocess
import time
from dataclasses import dataclass, field


@dataclass
class HpcOptions:
    """HPCdaligner's options (HPCdaligner.c:142-470), daligner's and LAmerge's among them."""
    verbose: int = 0
    bias: bool = False
    asymmetric: bool = False
    identity: bool = False
    ignore: bool = False
    k: int = 14
    w: int = 6
    h: int = 35
    t: int = 0
    H: int = 0
    e: float = 0.0
    m_rel: float = 0.0
    l: int = 1000
    s: int = 100
    M: int = 0
    no_trace: bool = False
    run_id: int = 1
    threads: int = 4
    masks: list = field(default_factory=list)
    dal: int = 4
    dal_diag: int = 0
    merge: int = 8
    consecutive: bool = False
    keep: bool = False
    sort: bool = False
    host: str | None = None
    port: int = 0
    merge_after: bool = False   # --run --merge: the plan's LAmerge calls after its daligner calls


def _diag_jobs(o: HpcOptions) -> int:
    # HPCdaligner.c:579-585
    if o.dal_diag == 0:
        return o.dal if o.host is None else 1
    return o.dal_diag


def plan(fblock: int, lblock: int, o: HpcOptions) -> list[tuple[int, list[int]]]:
    """The daligner calls as (A block, [B blocks in command-line order])."""
    jobs = []
    if o.consecutive:
        # block i against i..n (all blocks with -A), --dal per call (HPCdaligner.c:631-700)
        for i in range(fblock, lblock + 1):
            low = fblock if o.asymmetric else i
            hgh = lblock
            while low <= hgh:
                bl = []
                while low <= hgh and len(bl) < o.dal:
                    bl.append(low)
                    low += 1
                jobs.append((i, bl))
        return jobs
    # rounds: first the calls holding the diagonal, then --dal blocks further down each
    # round (HPCdaligner.c:702-790)
    dd = _diag_jobs(o)
    ncmp = (lblock - fblock + 1) * (lblock - fblock + 2) // 2
    cur, test, first = 0, 0, True
    while cur < ncmp:
        for i in range(fblock, lblock + 1):
            if first:
                hgh = i - test * dd
                low = max(fblock, hgh - dd + 1)
            else:
                hgh = i - (dd + (test - 1) * o.dal)
                low = max(fblock, hgh - o.dal + 1)
            if hgh >= low:
                jobs.append((i, list(range(hgh, low - 1, -1))))
                cur += hgh - low + 1
        first = False
        test += 1
    return jobs


def njobs(fblock: int, lblock: int, o: HpcOptions) -> int:
    """The job count HPCdaligner prints in its header (HPCdaligner.c:587-620)."""
    if o.consecutive:
        n = 0
        for i in range(fblock, lblock + 1):
            low = fblock if o.asymmetric else i
            hgh = lblock
            while low < hgh:
                c = 0
                while low <= hgh and c < o.dal:
                    c += 1
                    low += 1
                n += 1
        return n
    dd = _diag_jobs(o)
    return sum(1 + int(math.ceil(1.0 * max(i - fblock + 1 - dd, 0) / o.dal)) for i in range(fblock, lblock + 1))


def _fmt_g(x: float) -> str:
    return "%g" % x


def daligner_flags(o: HpcOptions, consecutive_order: bool) -> list[str]:
    """The daligner options of one plan line, in HPCdaligner's order."""
    f = []
    if o.verbose:
        f.append("-v")
    if o.bias:
        f.append("-b")
    if o.asymmetric:
        f.append("-A")
    if o.identity:
        f.append("-I")
    if o.ignore:
        f.append("-i")
    if o.k != 14:
        f.append(f"-k{o.k}")
    if o.w != 6:
        f.append(f"-w{o.w}")
    if o.h != 35:
        f.append(f"-h{o.h}")
    if o.t > 0:
        f.append(f"-t{o.t}")
    if o.H > 0:
        f.append(f"-H{o.H}")
    if o.e > .1:
        f.append("-e" + _fmt_g(o.e))
    if o.m_rel > .1:
        f.append("-m" + _fmt_g(o.m_rel))
    if o.l != 1000:
        f.append(f"-l{o.l}")
    if o.s != 100:
        f.append(f"-s{o.s}")
    # the reference prints the memory limit as -s (sic), before -T in -X order, after it otherwise
    if consecutive_order:
        if o.M > 0:
            f.append(f"-s{o.M}")
        if o.no_trace:
            f.append("-T")
    else:
        if o.no_trace:
            f.append("-T")
        if o.M > 0:
            f.append(f"-s{o.M}")
    if o.host:
        f.append(f"-D{o.host}" + (f":{o.port}" if o.port > 0 else ""))
    elif o.port > 0:
        f.append(f":{o.port}")
    f.append(f"-r{o.run_id}")
    f.append(f"-j{o.threads}")
    f.extend(f"-m{m}" for m in o.masks)
    return f


def exec_flags(o: HpcOptions) -> list[str]:
    """The options a plan line means, as `daligner_gpu` takes them (the plan text's -s for
    the memory limit is passed as -M here; -j is not needed on the GPU)."""
    if o.bias:
        raise ValueError("-b (biased k-mer sampling) is not supported by the GPU build")
    if o.ignore or o.host:
        raise ValueError("-i and -D are not supported by the GPU build")
    f = []
    if o.verbose:
        f.append("-v")
    if o.asymmetric:
        f.append("-A")
    if o.identity:
        f.append("-I")
    if o.k != 14:
        f.append(f"-k{o.k}")
    if o.w != 6:
        f.append(f"-w{o.w}")
    if o.h != 35:
        f.append(f"-h{o.h}")
    if o.t > 0:
        f.append(f"-t{o.t}")
    if o.H > 0:
        f.append(f"-H{o.H}")
    if o.e > .1:
        f.append("-e" + _fmt_g(o.e))
    if o.l != 1000:
        f.append(f"-l{o.l}")
    if o.s != 100:
        f.append(f"-s{o.s}")
    if o.M > 0:
        f.append(f"-M{o.M}")
    if o.no_trace:
        f.append("-T")
    f.append(f"-r{o.run_id}")
    f.extend(f"-m{m}" for m in o.masks)
    return f


def _db_parts(db: str):
    path = db if db.lower().endswith(".db") else db + ".db"
    name = os.path.basename(path)[:-3]
    d = os.path.dirname(path) or "."
    return path, name, d


def plan_text(db: str, fblock: int, lblock: int, o: HpcOptions) -> str:
    """HPCdaligner's plan as it prints it to stdout (daligner calls, then LAmerge calls)."""
    path, name, d = _db_parts(db)
    pre = (d if len(d) > 1 else "") + name
    out = [f"# Daligner jobs ({njobs(fblock, lblock, o)})"]
    flags = " ".join(daligner_flags(o, o.consecutive))
    for a, bl in plan(fblock, lblock, o):
        out.append(f"daligner {flags} {pre}.{a} " + " ".join(f"{pre}.{b}" for b in bl))
    out.append(f"# merge jobs({lblock - fblock + 1})")
    for i in range(fblock, lblock + 1):
        m = "LAmerge"
        if o.verbose:
            m += " -" + "v" * o.verbose
        if o.keep:
            m += " -k"
        if o.sort:
            m += " -s"
        m += f" -n {o.merge} {path} {name}.{i}.las %03d_%05d " % (o.run_id, i)
        out.append(m)
    return "\n".join(out) + "\n"


def db_blocks(db: str) -> int:
    """Number of blocks of a split DB (the `blocks =` line of the .db file)."""
    path, _, _ = _db_parts(db)
    with open(path) as f:
        for line in f:
            if line.startswith("blocks ="):
                return int(line.split("=")[1])
    return 1


def assign(jobs, world: int, rank: int):
    """This rank's share of the plan: longest-processing-time-first over the ranks by the
    number of block comparisons per call, ties by plan order.  Deterministic, so every rank
    computes the same split without communicating."""
    load = [0] * world
    mine = []
    order = sorted(range(len(jobs)), key=lambda j: (-len(jobs[j][1]), j))
    owner = {}
    for j in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[j] = r
        load[r] += len(jobs[j][1])
    for j in range(len(jobs)):
        if owner[j] == rank:
            mine.append(jobs[j])
    return mine


def cli_path() -> str:
    from . import build
    return build.CLI


def run_jobs(db: str, jobs, o: HpcOptions, executor=None):
    """Runs this rank's daligner calls in the DB's directory; returns (calls, seconds)."""
    path, name, d = _db_parts(db)
    flags = exec_flags(o)
    t0 = time.perf_counter()
    for a, bl in jobs:
        args = flags + [f"{name}.{a}"] + [f"{name}.{b}" for b in bl]
        if executor is not None:
            executor(d, args)
        else:
            exe = cli_path()
            if not os.path.exists(exe):
                raise RuntimeError(f"{exe} is missing: build it with `python marvel_b200/build.py`")
            subprocess.run([exe] + args, cwd=d, check=True)
    return len(jobs), time.perf_counter() - t0


def reduce_stats(calls: int, seconds: float):
    """(sum of calls, max of seconds) over the ranks of the default process group (or this
    process alone when none is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return calls, seconds
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    c = torch.tensor([float(calls)], dtype=torch.float64, device=dev)
    s = torch.tensor([seconds], dtype=torch.float64, device=dev)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.MAX)
    return int(c.item()), float(s.item())


def run_merges(db: str, blocks, o: HpcOptions, merger=None):
    """The plan's LAmerge calls for the given blocks: all .las files of run directory
    %03d_%05d (run id, block) merged into <db name>.<block>.las beside the DB, on the GPU."""
    path, name, d = _db_parts(db)
    for i in blocks:
        src = os.path.join(d, "%03d_%05d" % (o.run_id, i))
        out = os.path.join(d, f"{name}.{i}.las")
        if merger is not None:
            merger(src, out)
        else:
            from . import lamerge
            if lamerge.main(["-n", str(o.merge), path, out, src]) != 0:
                raise RuntimeError(f"merging {src} failed")
    return len(blocks)


def run(db: str, o: HpcOptions, fblock: int | None = None, lblock: int | None = None, executor=None, merge=False,
        merger=None):
    """Plans all block comparisons of db, runs this rank's share (rank and world from the
    default process group, if any), and returns (calls of all ranks, slowest rank's seconds).
    With merge, after all ranks finish their calls, each rank merges its share of the blocks
    (the plan's LAmerge calls)."""
    import torch.distributed as dist
    world, rank = 1, 0
    dist_on = dist.is_available() and dist.is_initialized()
    if dist_on:
        world, rank = dist.get_world_size(), dist.get_rank()
    n = db_blocks(db)
    fb = fblock or 1
    lb = lblock or n
    t0 = time.perf_counter()
    mine = assign(plan(fb, lb, o), world, rank)
    calls, _ = run_jobs(db, mine, o, executor)
    if merge:
        if dist_on:
            dist.barrier()   # every block's files are written before any merge reads them
        run_merges(db, list(range(fb, lb + 1))[rank::world], o, merger)
    return reduce_stats(calls, time.perf_counter() - t0)


def parse_args(argv):
    """HPCdaligner's command line -> (db, first block, last block, HpcOptions, run flag)."""
    import argparse
    p = argparse.ArgumentParser(prog="marvel_b200.hpc", add_help=False)
    p.add_argument("--run", action="store_true")
    p.add_argument("--merge", action="store_true")
    p.add_argument("-v", action="count", default=0)
    for c in "AIXTKS":
        p.add_argument("-" + c, action="store_true")
    for c, t in (("k", int), ("w", int), ("h", int), ("t", int), ("H", int), ("e", float), ("l", int),
                 ("s", int), ("M", int), ("r", int), ("j", int)):
        p.add_argument("-" + c, type=t)
    p.add_argument("-m", action="append", default=[])
    p.add_argument("--dal", type=int, default=4)
    p.add_argument("--dalDiag", type=int, default=0)
    p.add_argument("--mrg", type=int, default=8)
    p.add_argument("db")
    p.add_argument("blocks", nargs="?")
    a = p.parse_args(argv)
    o = HpcOptions(verbose=a.v, asymmetric=a.A, identity=a.I, consecutive=a.X, no_trace=a.T, keep=a.K, sort=a.S,
                   masks=a.m, dal=a.dal, dal_diag=a.dalDiag, merge=a.mrg)
    for c, f in (("k", "k"), ("w", "w"), ("h", "h"), ("t", "t"), ("H", "H"), ("e", "e"), ("l", "l"), ("s", "s"),
                 ("M", "M"), ("r", "run_id")):
        if getattr(a, c) is not None:
            setattr(o, f, getattr(a, c))
    if a.j is not None and a.j > 0 and (a.j & (a.j - 1)) == 0:  # powers of two only (HPCdaligner.c:264-277)
        o.threads = a.j
    n = db_blocks(a.db)
    fb, lb = 1, n
    if a.blocks:
        if "-" in a.blocks:
            fb, lb = (int(x) for x in a.blocks.split("-"))
        else:
            fb = lb = int(a.blocks)
    if fb < 1 or fb > n or lb < fb or lb > n:
        raise SystemExit(f"invalid block range {fb}-{lb} for a DB of {n} blocks")
    o.merge_after = a.merge
    return a.db, fb, lb, o, a.run


def main(argv=None):
    """python -m marvel_b200.hpc [--run [--merge]] [HPCdaligner options] DB [first[-last]]

    Without --run prints the plan like HPCdaligner.  With --run (one process per GPU, e.g.
    under torchrun) each rank runs its share of the daligner calls on its own GPU, and with
    --merge then its share of the LAmerge calls."""
    import sys
    db, fb, lb, o, do_run = parse_args(sys.argv[1:] if argv is None else argv)
    if not do_run:
        print(plan_text(db, fb, lb, o), end="")
        return 0
    import torch.distributed as dist
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        from datetime import timedelta
        local = int(os.environ.get("LOCAL_RANK", "0"))
        os.environ.setdefault("CUDA_VISIBLE_DEVICES", str(local))
        dist.init_process_group("gloo", timeout=timedelta(seconds=3600))
    calls, secs = run(db, o, fb, lb, merge=o.merge_after)
    if not dist.is_initialized() or dist.get_rank() == 0:
        print(f"{calls} daligner calls, slowest rank {secs:.1f} s")
    if dist.is_initialized():
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

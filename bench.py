#!/usr/bin/env python
"""bench.py -- overlaps/s of daligner's overlap path on B200.

A step is one daligner block comparison: one DB block against itself in both
orientations (Sort_Kmers(A), Match_Filter(A,A), complement_DB, Sort_Kmers(cA),
Match_Filter(A,cA), dalign/daligner.c:957-1012), on the bacterial-scale workload with
repeats (4.6 Mbp genome + 40 x 5 kbp repeats at 1.5% + 3 x 6 kbp at 0.2%, 25x PacBio-like
reads, mean 10 kbp; k14 w6 h35 e.70 l1000 s100 M32), generated from a seed.

  value  overlaps/s with the block resident in HBM (all device stages up to the overlap
         buffer sorted into .las order on the device; device-timed with CUDA events on the
         library's stream; nothing crosses PCIe inside the timed region)
  e2e    the same through the C ABI from pinned host buffers: block H2D + pipeline +
         sorted overlap buffer D2H, device-timed

Multi-GPU: each rank compares its own block (seed + rank): weak scaling, no collective on
the data path; the job value is all ranks' overlaps over the slowest rank's time.

--impl reference runs the reference daligner (built from source into oracle/_ref) on
the host cores (-j = the largest power of two <= cores) on the same block and flags, one
whole block comparison per step; cpu_baseline on the GPU line is one such run plus a
filter-only run, which split off the aligner's CPU time for its GCUPS.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from marvel_b200 import dazzdb, synth  # noqa: E402

PARAMS = dict(k=14, w=6, h=35, t=0, e=0.70, l=1000, s=100, M=32)
FLAGS = "-k14 -w6 -h35 -e.70 -l1000 -s100 -M32"
BIASED = False  # --biased: daligner -b on both arms


# a workload with two blocks generated compares block 1 against block 2, the rest one block
# against itself; synth.Workload.masks names the tracks daligner masks with (-m)
WORKLOAD = "cfg2"


def masks_of(workload=None):
    return list(synth.WORKLOADS[workload or WORKLOAD].masks)


def is_pair(workload=None):
    return synth.WORKLOADS[workload or WORKLOAD].nblocks >= 2


def flag_str():
    return ("-b " if BIASED else "") + "".join(f"-m{m} " for m in masks_of()) + FLAGS


def comparison():
    return "block 1 vs block 2" if is_pair() else "one block vs itself"


def path_name():
    return "daligner -b path" if BIASED else "plain daligner path"


CACHE = os.environ.get("MARVEL_B200_CACHE", os.path.join(tempfile.gettempdir(), "marvel_b200_bench"))
# k_align_pairs DRAM bytes (read + write) per wave cell, from the ncu capture of the cfg1
# N-orientation launch (profiles/k_align_pairs_cfg1.md): 85.0 MB over 282 M cells
ALIGN_DRAM_BYTES_PER_CELL = 84.96e6 / 282.0e6
# k-mer index build DRAM bytes per k-mer (extraction + 4 LSD passes), from the ncu capture of
# the cfg1 index (profiles/filter_kernels_cfg1.md): 1,731 MB over 21.08 M k-mers
INDEX_DRAM_BYTES_PER_KMER = 1731.2e6 / 21082465


def make_db(workload, seed_offset=0, scale=1.0):
    """Generates (or reuses) the DB of a workload; returns the path of block 1."""
    return synth.cached_db(workload, seed_offset, scale, CACHE)


def dust_track(path):
    """The dust track of the workload's DB (whole DB) for the reference arm, made once by the
    reference DBdust unless the GPU arm's device DBdust already wrote it (the same bytes)."""
    root = path.rsplit(".", 1)[0]
    if os.path.exists(os.path.join(os.path.dirname(root), "." + os.path.basename(root) + ".dust.anno")):
        return
    subprocess.run([ref_binary("DBdust"), os.path.basename(root)], cwd=os.path.dirname(root), check=True,
                   stdout=subprocess.DEVNULL)


def load_blocks(workload, seed_offset=0):
    """(A, B) of a workload: B is None for a block against itself; mask tracks loaded."""
    from marvel_b200 import workloads
    return workloads.blocks(workload, seed_offset, 1.0, CACHE)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_gpu(args):
    import torch
    import marvel_b200 as mb

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.synchronize()

    A, B = load_blocks(args.workload, seed_offset=rank)
    pair = B is not None
    free0, total_mem = torch.cuda.mem_get_info()
    ctx = mb.Context()
    p = PARAMS
    ctx.set_filter_params(p["k"], p["w"], p["t"], p["h"])
    ctx.new_align_spec(p["e"], p["s"], A.freq)
    ctx.set_globals(2 * p["l"], False, p["M"] * 0x40000000)
    ctx.set_biased(BIASED)
    if args.schedule or args.kinds:
        ctx.set_align_schedule([int(x) for x in args.schedule.split(",") if x],
                               [int(x) for x in args.kinds.split(",")] if args.kinds else None)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()

    def reduce(vals, op):
        if ws == 1:
            return vals
        t = torch.tensor(vals, dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=op)
        return t.tolist()

    # ---- device-resident timing
    ctx.load_block(0, A)
    if pair:
        ctx.load_block(1, B)
    tuned = None
    if args.autotune:
        from marvel_b200 import autotune
        tuned = autotune.tune(ctx, A, B)
    for _ in range(args.warmup):  # the same work as a timed step, so that every buffer is allocated
        ctx.reset_overlap_buffer()
        mb.run_loaded(ctx, not pair)
        ctx.sort_overlaps()
    barrier()
    l0 = mb.kernel_launches()
    times, recs = [], 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ctx.reset_overlap_buffer()
            ctx.timer_mark(0)
            mb.run_loaded(ctx, not pair)
            ctx.sort_overlaps()   # the .las order, on the device
            ctx.timer_mark(1)
            times.append(ctx.timer_elapsed_ms())
            recs += ctx.stats()["records"]
    barrier()
    launches = mb.kernel_launches() - l0
    st = ctx.stats()
    # device memory the library holds after the steps (its buffers are grown once and kept)
    held = free0 - torch.cuda.mem_get_info()[0]
    tot_ms = sum(times)
    tot_ms_max, = reduce([tot_ms], torch.distributed.ReduceOp.MAX if ws > 1 else None)
    recs_all, = reduce([float(recs)], torch.distributed.ReduceOp.SUM if ws > 1 else None)
    value = recs_all / (tot_ms_max / 1e3)

    # ---- end to end through the C ABI from pinned host buffers
    def pinned(X):
        pin = torch.empty(X.bases.size, dtype=torch.uint8, pin_memory=True)
        pin.numpy()[:] = X.bases
        return pin, dazzdb.Block(pin.numpy(), X.boff, X.rlen, X.ufirst, X.part, X.freq, X.maxlen, X.totlen,
                                 X.root, X.mask)
    pin_a, Ap = pinned(A)
    pin_b, Bp = pinned(B) if pair else (None, None)

    def block_bytes(X):
        n = X.bases.size + X.boff.nbytes + X.rlen.nbytes
        if X.mask is not None:
            n += 8 * (X.nreads + 1) + 8 * sum(len(iv) for iv in X.mask)
        return n
    h2d = block_bytes(A) + (block_bytes(B) if pair else 0)
    # result buffers in pinned host memory, sized from the device-resident runs
    nrec, ntb = ctx.sort_overlaps()
    pin_rec = torch.empty(int(nrec * 1.05 + 1024) * mb.OVL_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    pin_tr = torch.empty(int(ntb * 1.05 + 65536), dtype=torch.uint8, pin_memory=True)
    outbuf = (pin_rec.numpy().view(mb.OVL_DTYPE), pin_tr.numpy())
    etimes, erecs, d2h = [], 0, 0
    for i in range(args.warmup + args.steps):
        ctx.reset_overlap_buffer()
        ctx.timer_mark(0)
        ctx.load_block(0, Ap)
        if pair:
            ctx.load_block(1, Bp)
        mb.run_loaded(ctx, not pair)
        r, tr = ctx.overlaps(out=outbuf)
        ctx.timer_mark(1)
        if i >= args.warmup:
            etimes.append(ctx.timer_elapsed_ms())
            erecs += r.size
            d2h = r.size * mb.OVL_DTYPE.itemsize + tr.size
    barrier()
    e_ms_max, = reduce([sum(etimes)], torch.distributed.ReduceOp.MAX if ws > 1 else None)

    # ---- learned triage (beside the exact path): the shipped model, trained on another genome
    tri = None
    from marvel_b200 import triage as mtri
    model_path = args.triage_model or mtri.model_for(args.workload)
    if args.triage and os.path.exists(model_path):
        model = mtri.TriageModel.load(model_path)
        # one untimed plain run with collection: how the wave cells split between groups that
        # yield records and groups that do not (the most any triage can skip), and the
        # model's choices on those groups
        ctx.triage_reset()
        ctx.triage_collect(True)
        ctx.reset_overlap_buffer()
        mb.run_loaded(ctx, not pair)
        ctx.triage_collect(False)
        gfeat, grec, gcells = ctx.triage_groups()
        ctx.triage_reset()
        gprob = ctx.mlp_forward(model.params, gfeat)
        gev = mtri.evaluate(gprob, grec, gcells, model.threshold)
        dead = float(gcells[grec == 0].sum()) / max(float(gcells.sum()), 1.0)
        ctx.triage_set_model(model.params, model.threshold)
        ttimes, trecs, tskip, tgroups, talign = [], 0, 0, 0, 0.0
        for i in range(1 + args.steps):
            ctx.reset_overlap_buffer()
            ctx.timer_mark(0)
            mb.run_loaded(ctx, not pair)
            ctx.sort_overlaps()
            ctx.timer_mark(1)
            if i >= 1:
                ttimes.append(ctx.timer_elapsed_ms())
                tst = ctx.stats()
                trecs += tst["records"]
                tskip += sum(tst["skipped"])
                tgroups += sum(tst["groups"])
                talign += sum(tst["ms_align"])
        ctx.triage_set_model(None)
        barrier()
        t_ms_max, = reduce([sum(ttimes)], torch.distributed.ReduceOp.MAX if ws > 1 else None)
        trecs_all, = reduce([float(trecs)], torch.distributed.ReduceOp.SUM if ws > 1 else None)
        tri = {"value": round(trecs_all / (t_ms_max / 1e3), 1), "unit": "overlaps/s",
               "ms_per_step": round(t_ms_max / args.steps, 3),
               "record_recall": round(trecs / recs, 5) if recs else None,
               "groups_skipped": round(tskip / tgroups, 4) if tgroups else None,
               "seed_scan_align_ms": round(talign / args.steps, 3),
               "cells_skipped": round(gev["cells_skipped"], 4),
               "cells_in_groups_without_records": round(dead, 4),
               "bound": "skipping every group without records (and no other) would leave "
                        f"{1 - dead:.3f} of the wave cells: at most {1 / max(1 - dead, 1e-9):.2f}x on the aligner",
               "model": os.path.relpath(model_path, ROOT) + " (" + model_trained_on(model_path) + ")",
               "note": "records are a subset of the exact path's; recall < 1, so not the headline"}
    # ---- daligner2 (modimizer seeds) on the same resident block, beside the headline path
    d2 = None
    if args.d2:
        ctx.set_variant(2)
        ctx.set_filter_params(14, 6, 0, 35)
        ctx.load_block(0, A)
        d2times, d2recs = [], 0
        for i in range(1 + args.steps):
            ctx.reset_overlap_buffer()
            ctx.timer_mark(0)
            mb.run_loaded2(ctx, True)
            ctx.sort_overlaps()
            ctx.timer_mark(1)
            if i >= 1:
                d2times.append(ctx.timer_elapsed_ms())
                d2recs += ctx.stats()["records"]
        d2st = ctx.stats()
        ctx.set_variant(1)
        barrier()
        d2_ms, = reduce([sum(d2times)], torch.distributed.ReduceOp.MAX if ws > 1 else None)
        d2recs_all, = reduce([float(d2recs)], torch.distributed.ReduceOp.SUM if ws > 1 else None)
        d2 = {"value": round(d2recs_all / (d2_ms / 1e3), 1), "unit": "overlaps/s",
              "ms_per_step": round(d2_ms / args.steps, 3), "records_per_step": d2recs // args.steps,
              "stages_ms": {"index": round(d2st["ms_index"][0], 3), "merge_hitsort": round(sum(d2st["ms_merge"]), 3),
                            "seed_scan_align": round(sum(d2st["ms_align"]), 3)},
              "kmers": int(d2st["kmers"][0]), "hits": [int(x) for x in d2st["hits"]],
              "note": "daligner2 (dalign2/, modimizer seeds), same block and flags, device-resident like value"}
    erecs_all, = reduce([float(erecs)], torch.distributed.ReduceOp.SUM if ws > 1 else None)
    e2e = erecs_all / (e_ms_max / 1e3)

    out = None
    if rank == 0:
        ms_step = tot_ms_max / args.steps
        cells = sum(st["cells"])
        align_ms = sum(st["ms_align"])
        gcups = cells / (align_ms / 1e3) / 1e9 if align_ms > 0 else None
        peaks = load_peaks()
        clocks = clk.summary()
        # roofline of the dominant stage: the seed-scan/alignment kernel is integer-issue bound;
        # its algorithmic work is 16 integer lane-ops per wave cell (the reference's per-cell
        # body, dalign/align.c:748-910).  Peak = 148 SMs x 4 schedulers x 32 lanes x SM clock.
        sm_hz = (clocks["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)) * 1e6
        issue_peak = 148 * 128 * sm_hz / 1e12  # T lane-ops/s
        achieved = cells * 16 / (align_ms / 1e3) / 1e12 if align_ms > 0 else None
        kmers = sum(st["kmers"][0:3:2])
        idx_ms = st["ms_index"][0] + st["ms_index"][2]
        # k-mer index: extraction writes 8 B per k-mer and reads 1 B/base; 4 LSD passes move
        # 16 B per k-mer each (read+write key and value), as the reference's pass count
        idx_bytes = kmers * (8 + 1 + 4 * 16 + 12)
        out = {
            "metric": f"overlaps/s ({path_name()}, {comparison()})",
            "value": round(value, 1),
            "unit": "overlaps/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_step, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u8/int32",
            "data": "synthetic (seeded generator, no dataset)",
            "config": bench_config(args, A, ws, B),
            "records_per_step": recs // args.steps,
            "stages_ms": {"index": round(idx_ms, 3), "merge_hitsort": round(sum(st["ms_merge"]), 3),
                          "seed_scan_align": round(align_ms, 3)},
            "gcups": round(gcups, 2) if gcups else None,
            # the last step's aligner work (both orientations): pair groups aligned, those whose
            # band outgrew the 128-diagonal instance (redone on the wide one), seeds, wave cells
            "aligner": {"pair_groups": int(sum(st["groups"])), "wide_groups": int(sum(st["wide"])),
                        "seeds": int(sum(st["seeds"])), "wave_cells": int(sum(st["cells"]))},
            # per-stage rates of the last step (its stats): k-mers sorted, hits emitted and
            # sorted, Local_Alignment calls
            "rates": {"kmers_sorted_per_s": round(kmers / (idx_ms / 1e3), 1) if idx_ms > 0 else None,
                      "hits_per_s": round(sum(st["hits"]) / (sum(st["ms_merge"]) / 1e3), 1)
                      if sum(st["ms_merge"]) > 0 else None,
                      "alignments_per_s": round(sum(st["seeds"]) / (align_ms / 1e3), 1) if align_ms > 0 else None},
            "roofline": {"bound": "issue", "kernel": "k_align_pairs", "achieved": round(achieved, 3),
                         "peak": round(issue_peak, 2), "unit": "T int lane-ops/s",
                         "frac": round(achieved / issue_peak, 4),
                         "traffic": int(ALIGN_DRAM_BYTES_PER_CELL * cells / 2),
                         "traffic_source": "bytes per launch: dram read+write per wave cell of the cfg1 ncu capture "
                                           "(profiles/k_align_pairs_cfg1.md) x this launch's cells",
                         "peak_source": "derived: 148 SM x 128 lanes/clk x median SM clock under load",
                         "issue_slots_busy": 0.781,
                         "issue_source": "smsp__issue_active of the cfg1 ncu capture (profiles/k_align_pairs_cfg1.md): "
                                         "the kernel issues on 78 % of cycles; a wave is ~11 diagonals wide, so a "
                                         "warp instruction carries about a third of a warp of cells"},
            "roofline_filter": {"bound": "hbm", "kernel": "k-mer index (extract + 4 LSD passes)",
                                "achieved": round(idx_bytes / (idx_ms / 1e3) / 1e9, 1),
                                "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                                "frac": round(idx_bytes / (idx_ms / 1e3) / 1e9 / peaks.get("hbm_gbs", 6650.0), 4),
                                "traffic": int(INDEX_DRAM_BYTES_PER_KMER * kmers),
                                "traffic_source": "dram read+write per k-mer of the cfg1 index build's ncu capture "
                                                  "(profiles/filter_kernels_cfg1.md) x this step's k-mers",
                                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
            "e2e": {"value": round(e2e, 1), "unit": "overlaps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "device_gb_held": round(held / 1e9, 2),
            "device_gb_total": round(total_mem / 1e9, 1),
            "align_schedule": (("one launch per length class, alen+blen edges " + args.schedule) if args.schedule
                               else (f"autotuned: {tuned['chosen']}" if tuned
                                     else "one persistent launch, pair groups longest first from a device queue"))
            + (f"; instances {args.kinds} (0 warp, 1 wide, 2 duo)" if args.kinds else ""),
            "autotune": tuned,
            "triage": tri,
            "daligner2": d2,
            "clocks": clocks,
        }
        if args.cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args, cells)
            if d2 is not None and ref_binary("daligner2"):
                j = ref_threads()
                n2, dt2 = run_reference_once(make_db(args.workload), j, prog="daligner2")
                d2["cpu_baseline"] = {"value": round(n2 / dt2, 1), "unit": "overlaps/s", "cores": j,
                                      "kind": "reference",
                                      "sample": f"reference daligner2 -T{j} on the same block ({n2} overlaps, "
                                                f"{dt2:.1f} s wall)"}
        print(json.dumps(out), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return out


WORKLOAD_DESC = {
    "cfg2": "4.6 Mbp random genome + 40x5 kbp repeats @1.5% + 3x6 kbp @0.2%, 25x reads, log-normal mean 10 kbp "
            "sd 5 kbp, 9/4.5/1.5% ins/del/sub; one block (~115 Mbp) vs itself",
    "cfg1": "1 Mbp genome, 20x, mean 8 kbp sd 4 kbp, 9/4.5/1.5% ins/del/sub; one block vs itself",
    "cfg3": "10 Mbp genome, 30x, mean 20 kbp sd 15 kbp (1-150 kbp), 3/5/2% ins/del/sub; one block vs itself",
    "cfg4": "20 Mbp genome, 10% interspersed 1-8 kbp repeat families at 5-15% divergence, 30x, mean 10 kbp; "
            "block 1 (200 Mbp) vs itself",
    "cfg5": "200 Mbp diploid (0.5% SNP, 0.05% indel), 35% interspersed 1-10 kbp repeats at 5-15%, 2% tandem "
            "repeats, 30x, mean 15 kbp; 400 Mbp block 1 vs 400 Mbp block 2 with -mdust",
}


def model_trained_on(model_path):
    try:
        with open(os.path.splitext(model_path)[0] + ".json") as f:
            return "trained on the GPU on " + json.load(f)["trained_on"]
    except (OSError, KeyError, ValueError):
        return "trained on the GPU"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def ref_binary(prog="daligner"):
    b = os.path.join(ROOT, "oracle", "_ref", prog)
    return b if os.path.exists(b) and os.access(b, os.X_OK) else None


def ref_threads():
    n = os.cpu_count() or 1
    j = 1
    while j * 2 <= n:
        j *= 2
    return j


def run_reference_once(path, threads, h=35, prog="daligner"):
    """The reference daligner (or daligner2) on the workload's comparison (a block against
    itself, or block 1 against block 2 with its mask tracks); returns (records written,
    seconds).  With h=100000 no pair group reaches the aligner: the filter alone."""
    b = ref_binary(prog)
    d = os.path.dirname(path)
    name = os.path.basename(path)
    bname = name[:-2] + ".2" if is_pair() else name
    masks = [f"-m{m}" for m in masks_of()]
    if masks:
        dust_track(path)
    if prog == "daligner2":
        cmd = [b, f"-T{threads}", "-Pd2out", "-M32", "-k14", "-w6", f"-h{h}", "-e.70", "-l1000", "-s100", name, name]
        las = [os.path.join(d, "d2out_00001", "W.1.W.1.las")]
    else:
        cmd = [b, f"-j{threads}"] + (["-b"] if BIASED else []) + masks + ["-M32", "-k14", "-w6", f"-h{h}", "-e.70",
                                                                          "-l1000", "-s100", name, bname]
        las = [os.path.join(d, "001_00001", "W.1.W.2.las"), os.path.join(d, "001_00002", "W.2.W.1.las")] \
            if is_pair() else [os.path.join(d, "001_00001", "W.1.W.1.las")]
    t = time.perf_counter()
    subprocess.run(cmd, cwd=d, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    dt = time.perf_counter() - t
    n = 0
    for x in las:
        with open(x, "rb") as f:
            n += int(np.frombuffer(f.read(8), "<i8")[0])
    return n, dt


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def bench_config(args, A, ws, B=None):
    """The workload both arms run (the same dict on both JSON lines)."""
    out = {"workload": f"{args.workload}: " + WORKLOAD_DESC.get(args.workload, args.workload),
           "flags": flag_str(), "block_reads": int(A.nreads), "block_bases": int(A.totlen),
           "parallelism": f"dp{ws} (one block {'pair' if B is not None else ''} per rank)".replace("  ", " "),
           "l2": "inputs larger than L2 (k-mer index > 1 GB)"}
    if B is not None:
        out["b_block_reads"] = int(B.nreads)
        out["b_block_bases"] = int(B.totlen)
    return out


def pinned_cells(workload):
    """The reference's own wave-cell count for the full block of a workload (its WAVE_STATS
    counters), as recorded beside the parity digests; None when not recorded."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "config_digests.json")) as f:
            rec = json.load(f).get(workload)
    except OSError:
        return None
    if rec and rec.get("scale") == 1.0 and rec.get("seed_offset") == 0:
        return rec.get("cells")
    return None


def cpu_baseline(args, cells=None):
    """The reference daligner on the host cores, on the same block as the GPU arm: one full
    run and one filter-only run (-h100000: no pair group reaches the aligner), so that the
    aligner's CPU time and its GCUPS (the same wave cells the GPU counts, equal to the
    reference's WAVE_STATS count) follow."""
    path = make_db(args.workload)
    if ref_binary():
        j = ref_threads()
        n, dt = run_reference_once(path, j)
        _, df = run_reference_once(path, j, h=100000)
        out = {"value": round(n / dt, 1), "unit": "overlaps/s", "cores": j, "kind": "reference",
               "sample": f"reference daligner -j{j} on the same block as the GPU arm ({n} overlaps, {dt:.1f} s wall)",
               "filter_only_s": round(df, 2), "cpu_model": cpu_model()}
        if cells and dt > df:
            out["align_s"] = round(dt - df, 2)
            out["gcups"] = round(cells / (dt - df) / 1e9, 3)
            out["gcups_source"] = ("wave cells of the block (the GPU's count, equal to the reference's WAVE_STATS "
                                   "count) / (full run - filter-only run) wall time")
        return out
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    A, B = load_blocks(args.workload)
    p = oracle.make_params(A.freq)
    t = time.perf_counter()
    Bx = A if B is None else B
    recs, _, _ = oracle.daligner(A, Bx, dazzdb.complement_block(Bx), p, B is None)
    dt = time.perf_counter() - t
    return {"value": round(len(recs) / dt, 1), "unit": "overlaps/s", "cores": 1, "kind": "port",
            "sample": f"C restatement, 1 thread, on the same block as the GPU arm"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return None
    if not ref_binary():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/daligner was not built "
                          "(make -C oracle ref needs the reference sources)"}))
        return None
    path = make_db(args.workload)
    A = dazzdb.open_block(path)
    B = dazzdb.open_block(path[:-2] + ".2") if is_pair() else None
    j = ref_threads()
    for _ in range(args.warmup):
        run_reference_once(path, j)
    n_tot, t_tot = 0, 0.0
    for _ in range(args.steps):
        n, dt = run_reference_once(path, j)
        n_tot += n
        t_tot += dt
    v = n_tot / t_tot
    sample = (f"reference daligner -j{j} (host cores, {cpu_model()}) on the same block as the GPU arm, "
              f"{n_tot // args.steps} overlaps per step")
    out = {"impl": "reference", "metric": f"overlaps/s ({path_name()}, {comparison()})",
           "value": round(v, 1), "unit": "overlaps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1e3 * t_tot / args.steps, 1), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic (seeded generator, no dataset)",
           "config": bench_config(args, A, ws, B),
           "cpu_baseline": {"value": round(v, 1), "unit": "overlaps/s", "cores": j, "kind": "reference",
                            "sample": sample},
           "e2e": {"value": round(v, 1), "unit": "overlaps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    cells = pinned_cells(args.workload)
    if cells and not BIASED:
        out["gcups_whole_run"] = round(cells / (t_tot / args.steps) / 1e9, 3)
        out["gcups_note"] = ("the reference's WAVE_STATS wave cells of this block over the whole run's wall time "
                             "(filter included); bench.py's GPU line splits the filter off")
    print(json.dumps(out), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=sorted(synth.WORKLOADS))
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-triage", dest="triage", action="store_false",
                    help="skip the learned-triage measurement (reported beside the exact path)")
    ap.add_argument("--triage-model", default=None, help="model file (default: the shipped model)")
    ap.add_argument("--autotune", action="store_true",
                    help="time the aligner schedules on the block first and run the fastest (marvel_b200.autotune)")
    ap.add_argument("--schedule", default="",
                    help="alen+blen edges (bp, comma-separated): one aligner launch per length class instead of "
                         "the one persistent launch (a comparison schedule)")
    ap.add_argument("--kinds", default="",
                    help="the aligner instance of each length class (comma-separated, longest class first; one "
                         "entry without --schedule): 0 warp, 1 wide, 2 duo")
    ap.add_argument("--no-d2", dest="d2", action="store_false",
                    help="skip the daligner2 (modimizer seeds) measurement (reported beside the exact path)")
    ap.add_argument("--biased", action="store_true",
                    help="daligner -b (frequency-weighted tuples) on both arms instead of the plain path")
    args = ap.parse_args()
    global BIASED, WORKLOAD
    BIASED = args.biased
    WORKLOAD = args.workload
    if is_pair():
        args.d2 = False  # the daligner2 line is measured on the one-block workloads
    if BIASED:
        args.d2 = False  # daligner2 has no -b
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

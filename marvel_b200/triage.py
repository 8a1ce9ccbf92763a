"""Learned triage of pair groups: collection, GPU training, calibration, and the model file.

The aligner (report_thread, dalign/filter.c:1656-1995) aligns every pair group of an A read
and a B read in one orientation that has at least ceil(h/k) hits.  Most of the groups in a
repetitive genome yield no overlap, yet each costs wave cells.  The triage predicts, from
12 features of a group's hits, whether the plain path would emit a record for it and skips
the groups below a threshold.  A group is aligned or skipped as a whole, so every record
of the triaged path is a record of the plain path; what the triage can lose is recall,
which the threshold bounds (``calibrate``).

Features (one row per group, computed on the device inside Match_Filter):
  f0 log2 #hits, f1 log2 |A|, f2 log2 |B|, f3 apos span / |A|, f4 log2(1 + diagonal range),
  f5 mean diagonal / |A|, f6 log2(1 + diagonal sd), f7 overlap length on the mean diagonal
  / (2 * minover), f8 hits per 64 bp of apos span, f9 fraction of hits within one band
  (2^w) of the mean diagonal, f10 orientation, f11 masked fraction of the A read.

Model: 12-64-64-1 ReLU MLP; forward, backward and Adam run as BF16 tensor-core kernels with
FP32 accumulation and FP32 optimizer state (libgpudalign.so, gd_triage.cu).
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import TRI_NF, TRI_NPARAM, Context, _check, lib, run_loaded

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "models", "triage_cfg12.npz")
# the training blocks of the default model: the CPU-runnable and the bacterial-scale
# workloads' models on other seeds than the benchmark's (seed offset 0), about 10^7 groups
TRAIN_SPECS = (("cfg2", 1), ("cfg2", 2), ("cfg1", 1), ("cfg1", 2), ("cfg1", 3), ("cfg1", 4))


@dataclass
class TriageModel:
    params: np.ndarray   # TRI_NPARAM float32 (gd_triage_set_model layout)
    threshold: float     # groups with predicted probability below this are skipped
    recall: float        # record recall the threshold was calibrated for

    def save(self, path):
        np.savez(path, params=self.params, threshold=np.float32(self.threshold), recall=np.float32(self.recall))

    @staticmethod
    def load(path) -> "TriageModel":
        z = np.load(path)
        return TriageModel(np.asarray(z["params"], np.float32), float(z["threshold"]), float(z["recall"]))


def model_for(workload: str) -> str:
    """The shipped model for a workload: the default weights with the threshold calibrated on
    another genome of that workload's model when such a file exists (triage_cfg12_cal_<w>.npz),
    else the default model."""
    cal = os.path.join(HERE, "models", f"triage_cfg12_cal_{workload}.npz")
    return cal if os.path.exists(cal) else DEFAULT_MODEL


def mlp_init(feat: np.ndarray, seed: int = 1) -> np.ndarray:
    """Feature scales from feat and seeded He-uniform weights (gd_mlp_init)."""
    feat = np.ascontiguousarray(feat, np.float32).reshape(-1, TRI_NF)
    params = np.zeros(TRI_NPARAM, np.float32)
    _check(lib().gd_mlp_init(feat.ctypes.data, feat.shape[0], C.c_uint64(seed), params.ctypes.data))
    return params


def collect(ctx: Context, blocks, self_cmp=True):
    """Runs the plain path over the given loaded-block callbacks with collection on and
    returns (features, records per group, cells per group).  blocks is an iterable of
    callables that load the slots of one comparison into ctx (the caller sets the
    parameters, as daligner_block does)."""
    ctx.triage_reset()
    ctx.triage_collect(True)
    try:
        for load in blocks:
            load()
            run_loaded(ctx, self_cmp)
    finally:
        ctx.triage_collect(False)
    return ctx.triage_groups()


def labels(records: np.ndarray) -> np.ndarray:
    return (np.asarray(records) > 0).astype(np.float32)


def train(ctx: Context, feat, records, *, epochs=30, batch=4096, lr=3e-3, pos_weight=None, seed=1):
    """Trains the MLP on the device; pos_weight defaults to #negatives / #positives so that a
    missed positive costs as much as all negatives together on average."""
    y = labels(records)
    npos = float(y.sum())
    if pos_weight is None:
        pos_weight = max(1.0, (len(y) - npos) / max(npos, 1.0))
    params = mlp_init(feat, seed)
    params, losses = ctx.mlp_train(feat, y, params, epochs=epochs, batch=batch, lr=lr, pos_weight=pos_weight,
                                   seed=seed)
    return params, losses


def calibrate(prob: np.ndarray, records: np.ndarray, recall: float = 0.999) -> float:
    """The largest threshold whose skipped groups hold at most (1 - recall) of the records
    (record-weighted recall on the calibration rows).  Groups without records never limit it."""
    prob = np.asarray(prob, np.float64)
    rec = np.asarray(records, np.float64)
    total = rec.sum()
    if total == 0:
        return 0.0
    budget = (1.0 - recall) * total
    order = np.argsort(prob, kind="stable")
    lost = np.cumsum(rec[order])
    # skipping order[:i] loses lost[i-1]; allow i groups while lost stays within budget
    i = int(np.searchsorted(lost, budget, side="right"))
    if i >= len(order):
        return float(np.nextafter(np.float32(prob.max()), np.float32(np.inf)))
    # threshold at the first group that must be kept; ties with it are kept too
    return float(prob[order[i]])


def evaluate(prob, records, cells, threshold):
    """Record recall, skipped-group fraction and skipped-cell fraction at threshold."""
    prob = np.asarray(prob)
    rec = np.asarray(records, np.float64)
    cells = np.asarray(cells, np.float64)
    skip = prob < threshold
    total = rec.sum()
    return {
        "recall": float(1.0 - rec[skip].sum() / total) if total else 1.0,
        "groups_skipped": float(skip.mean()) if len(skip) else 0.0,
        "cells_skipped": float(cells[skip].sum() / cells.sum()) if cells.sum() else 0.0,
    }


def fit(ctx: Context, feat, records, *, recall=0.999, holdout=0.25, seed=1, **kw) -> tuple[TriageModel, dict]:
    """Trains on part of the rows and calibrates the threshold on the held-out rest."""
    n = len(records)
    rng = np.random.default_rng(seed)
    idx = rng.permutation(n)
    nh = int(n * holdout)
    cal, tr = idx[:nh], idx[nh:]
    params, losses = train(ctx, feat[tr], records[tr], seed=seed, **kw)
    pc = ctx.mlp_forward(params, feat[cal])
    thr = calibrate(pc, records[cal], recall)
    info = {"losses": losses.tolist(), "calibration": evaluate(pc, records[cal], np.ones(len(cal)), thr)}
    return TriageModel(params, thr, recall), info


def train_on_workload(workload: str, seed_offset: int, out: str, recall: float = 0.999, epochs: int = 25,
                      scale: float = 1.0, batch: int = 8192):
    """Collects the groups of one synthetic block compared with itself (bench's generator,
    another seed than the benchmark's), trains on the device and writes the model file."""
    return train_on_workloads(((workload, seed_offset),), out, recall, epochs, scale, batch)


def train_on_workloads(specs, out: str, recall: float = 0.999, epochs: int = 25, scale: float = 1.0,
                       batch: int = 8192):
    """Collects the groups of synthetic blocks, each compared with itself -- specs lists
    (workload, seed offset) pairs, seed offsets other than the benchmark's 0 -- trains on
    the device with mini-batches of batch groups and writes the model file and a .json
    record of the training."""
    import json
    import time

    from . import daligner_block, dazzdb, synth

    ctx = Context()
    feats, recs = [], []
    for workload, seed_offset in specs:
        A = dazzdb.open_block(synth.cached_db(workload, seed_offset, scale))
        ctx.triage_reset()
        ctx.triage_collect(True)
        daligner_block(ctx, A)
        ctx.triage_collect(False)
        feat, rec, _ = ctx.triage_groups()
        feats.append(feat)
        recs.append(rec)
    feat = np.concatenate(feats)
    rec = np.concatenate(recs)
    t0 = time.perf_counter()
    model, info = fit(ctx, feat, rec, recall=recall, epochs=epochs, batch=batch)
    info["train_s"] = round(time.perf_counter() - t0, 2)
    info["groups"] = int(len(rec))
    info["positive_groups"] = int((rec > 0).sum())
    info["batch"] = batch
    info["epochs"] = epochs
    info["trained_on"] = ", ".join(f"{w} genome seed offset {o}" for w, o in specs) + f" (scale {scale}); the "
    info["trained_on"] += "benchmark's blocks are seed offset 0"
    ctx.close()
    model.save(out)
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump({k: v for k, v in info.items() if k != "losses"} | {"final_loss": info["losses"][-1]}, f, indent=1)
    return model, info


def calibrate_on_workload(model_path: str, workload: str, seed_offset: int, out: str, recall: float = 0.999):
    """Keeps a model's weights and re-calibrates its threshold on the pair groups of another
    genome of a workload's model (seed offset other than the benchmark's 0): the largest
    threshold whose skipped groups hold at most 1 - recall of that genome's records.  Writes
    the model file and a .json record."""
    import json

    from . import daligner_block, workloads

    model = TriageModel.load(model_path)
    A, B = workloads.blocks(workload, seed_offset)
    ctx = Context()
    ctx.triage_reset()
    ctx.triage_collect(True)
    daligner_block(ctx, A, B)
    ctx.triage_collect(False)
    feat, rec, cells = ctx.triage_groups()
    prob = ctx.mlp_forward(model.params, feat)
    ctx.close()
    thr = calibrate(prob, rec, recall)
    cal = TriageModel(model.params, thr, recall)
    cal.save(out)
    info = {"weights": os.path.basename(model_path), "calibrated_on": f"{workload} genome seed offset {seed_offset}",
            "groups": int(len(rec)), "positive_groups": int((rec > 0).sum()), "threshold": thr,
            "at_threshold": evaluate(prob, rec, cells, thr),
            "at_training_threshold": evaluate(prob, rec, cells, model.threshold)}
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    return cal, info


def main(argv=None):
    """python -m marvel_b200.triage train [--workload cfg2:1 ...] [--batch 8192] [--out PATH]
    python -m marvel_b200.triage calibrate --model PATH --workload cfg5:1 [--recall 0.999] --out PATH"""
    import argparse
    p = argparse.ArgumentParser(prog="marvel_b200.triage")
    p.add_argument("cmd", choices=["train", "calibrate"])
    p.add_argument("--model", default=DEFAULT_MODEL, help="calibrate: the model whose weights are kept")
    p.add_argument("--workload", action="append", help="workload:seed_offset (repeatable); default: TRAIN_SPECS")
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--recall", type=float, default=0.999)
    p.add_argument("--epochs", type=int, default=25)
    p.add_argument("--batch", type=int, default=8192)
    p.add_argument("--out", default=DEFAULT_MODEL)
    a = p.parse_args(argv)
    specs = [(w.split(":")[0], int(w.split(":")[1])) for w in a.workload] if a.workload else TRAIN_SPECS
    if a.cmd == "calibrate":
        if len(specs) != 1 or not a.workload:
            p.error("calibrate takes one --workload NAME:SEED_OFFSET")
        cal, info = calibrate_on_workload(a.model, specs[0][0], specs[0][1], a.out, a.recall)
        print(f"threshold {cal.threshold:.4g}; {info['at_threshold']}; at the training threshold "
              f"{info['at_training_threshold']}")
        return 0
    model, info = train_on_workloads(specs, a.out, a.recall, a.epochs, a.scale, a.batch)
    print(f"threshold {model.threshold:.4g}; calibration {info['calibration']}; {info['train_s']} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

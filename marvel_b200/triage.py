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
from dataclasses import dataclass

import numpy as np

from . import TRI_NF, TRI_NPARAM, Context, _check, lib, run_loaded


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

"""marvel_b200 -- daligner's overlap path on B200 (sm_100a), behind a C ABI.

The product is ``libgpudalign.so`` (CUDA kernels + host orchestration, ``include/gpudalign.h``)
and the ``daligner_gpu`` command-line driver.  This module is the thin Python binding used
by tests and benchmarks: it loads the in-tree shared library with ctypes and exposes the
reference's operator interface of the path (dalign/filter.h:67-73, dalign/align.h:160-344):

    ctx = Context()
    ctx.set_filter_params(k, w, t, h)          # Set_Filter_Params
    ctx.new_align_spec(e, s, freq, ...)        # New_Align_Spec
    ctx.load_block(slot, block); ctx.sort_kmers(slot)    # Sort_Kmers
    ctx.match_filter(bslot, comp, self)        # Match_Filter
    ctx.write_overlap_buffer(...)              # Write_Overlap_Buffer

There is no CPU path: without a CUDA device ``Context()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import dazzdb

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libgpudalign.so")
_lib = None


class GdBlock(C.Structure):
    _fields_ = [("bases", C.c_void_p), ("boff", C.c_void_p), ("rlen", C.c_void_p), ("nreads", C.c_int32),
                ("maxlen", C.c_int32), ("totlen", C.c_int64), ("ufirst", C.c_int32),
                ("mask_anno", C.c_void_p), ("mask_data", C.c_void_p)]


class GdOverlap(C.Structure):
    _fields_ = [("tlen", C.c_int32), ("diffs", C.c_int32), ("abpos", C.c_int32), ("bbpos", C.c_int32),
                ("aepos", C.c_int32), ("bepos", C.c_int32), ("flags", C.c_uint32), ("aread", C.c_int32),
                ("bread", C.c_int32), ("pad", C.c_int32), ("toff", C.c_uint64)]


OVL_DTYPE = np.dtype([("tlen", "<i4"), ("diffs", "<i4"), ("abpos", "<i4"), ("bbpos", "<i4"), ("aepos", "<i4"),
                      ("bepos", "<i4"), ("flags", "<u4"), ("aread", "<i4"), ("bread", "<i4"), ("pad", "<i4"),
                      ("toff", "<u8")])
assert OVL_DTYPE.itemsize == C.sizeof(GdOverlap)


class GdStats(C.Structure):
    _fields_ = [("kmers", C.c_int64 * 3), ("hits", C.c_int64 * 2), ("groups", C.c_int64 * 2),
                ("seeds", C.c_int64 * 2), ("cells", C.c_int64 * 2), ("records", C.c_int64),
                ("limit", C.c_int32 * 2), ("ms_index", C.c_double * 3), ("ms_merge", C.c_double * 2),
                ("ms_align", C.c_double * 2), ("skipped", C.c_int64 * 2), ("wide", C.c_int64 * 2),
                ("reruns", C.c_int64 * 2)]


# exported symbols of include/gpudalign.h
SYMBOLS = ["gd_create", "gd_destroy", "gd_last_error", "gd_set_filter_params", "gd_new_align_spec",
           "gd_set_globals", "gd_load_block", "gd_sort_kmers", "gd_get_kmers", "gd_match_filter", "gd_get_hits",
           "gd_num_overlaps", "gd_get_overlaps", "gd_write_overlap_buffer", "gd_reset_overlap_buffer",
           "gd_get_stats", "gd_local_alignment_batch", "gd_complement_block", "gd_timer_mark",
           "gd_timer_elapsed_ms", "gd_kernel_launches", "gd_local_alignment_batch_noalloc",
           "gd_compute_trace_pts", "gd_triage_collect", "gd_triage_get_groups", "gd_triage_reset",
           "gd_triage_set_model", "gd_mlp_init", "gd_mlp_forward", "gd_mlp_grad", "gd_mlp_train", "gd_sort_overlaps", "gd_las_sort", "gd_dust", "gd_las_merge",
           "gd_set_wave_limit", "gd_set_variant", "gd_match_filter2", "gd_test_handle_redundancies_d2",
           "gd_set_biased", "gd_set_capacities", "gd_test_wait_expiry", "gd_set_align_schedule"]

TRI_NF = 12        # features per pair group
TRI_NPARAM = 5081  # model parameter vector (gd_triage_set_model)


def lib():
    """Loads the in-tree libgpudalign.so (built by marvel_b200/build.py); fails loudly if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"{LIBPATH} is missing: build it with `python marvel_b200/build.py`")
    L = C.CDLL(LIBPATH)
    L.gd_create.restype = C.c_void_p
    L.gd_destroy.argtypes = [C.c_void_p]
    L.gd_last_error.restype = C.c_char_p
    L.gd_set_filter_params.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    L.gd_new_align_spec.argtypes = [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int]
    L.gd_set_globals.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64]
    L.gd_load_block.argtypes = [C.c_void_p, C.c_int, C.POINTER(GdBlock)]
    L.gd_set_variant.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.gd_set_biased.argtypes = [C.c_void_p, C.c_int]
    L.gd_match_filter2.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.gd_sort_kmers.argtypes = [C.c_void_p, C.c_int]
    L.gd_sort_kmers.restype = C.c_int64
    L.gd_get_kmers.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    L.gd_get_kmers.restype = C.c_int64
    L.gd_match_filter.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.gd_get_hits.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    L.gd_get_hits.restype = C.c_int64
    L.gd_num_overlaps.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.gd_num_overlaps.restype = C.c_int64
    L.gd_get_overlaps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]
    L.gd_get_overlaps.restype = C.c_int64
    L.gd_sort_overlaps.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.gd_sort_overlaps.restype = C.c_int64
    L.gd_las_sort.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
    L.gd_las_sort.restype = C.c_int64
    L.gd_las_merge.argtypes = [C.c_void_p, C.POINTER(C.c_char_p), C.c_int, C.c_char_p]
    L.gd_las_merge.restype = C.c_int64
    L.gd_set_wave_limit.argtypes = [C.c_void_p, C.c_int]
    L.gd_set_capacities.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64]
    L.gd_test_wait_expiry.argtypes = [C.c_void_p, C.c_int]
    L.gd_set_align_schedule.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.gd_dust.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_float),
                          C.c_void_p, C.c_void_p, C.c_int64]
    L.gd_dust.restype = C.c_int64
    L.gd_write_overlap_buffer.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    L.gd_reset_overlap_buffer.argtypes = [C.c_void_p]
    L.gd_get_stats.argtypes = [C.c_void_p, C.POINTER(GdStats)]
    L.gd_local_alignment_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                           C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.gd_complement_block.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.gd_timer_mark.argtypes = [C.c_void_p, C.c_int]
    L.gd_timer_elapsed_ms.argtypes = [C.c_void_p]
    L.gd_timer_elapsed_ms.restype = C.c_double
    L.gd_kernel_launches.restype = C.c_ulonglong
    L.gd_compute_trace_pts.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_void_p]
    L.gd_local_alignment_batch_noalloc.argtypes = [C.c_void_p] + [C.c_void_p] * 8 + [C.c_int] * 3 + \
        [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.gd_triage_collect.argtypes = [C.c_void_p, C.c_int]
    L.gd_triage_get_groups.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    L.gd_triage_get_groups.restype = C.c_int64
    L.gd_triage_reset.argtypes = [C.c_void_p]
    L.gd_triage_set_model.argtypes = [C.c_void_p, C.c_void_p, C.c_float]
    L.gd_mlp_init.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p]
    L.gd_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    L.gd_mlp_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p,
                              C.c_void_p]
    L.gd_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_float,
                               C.c_float, C.c_uint64, C.c_void_p, C.c_void_p]
    _lib = L
    return L


def kernel_launches():
    """Kernels libgpudalign.so has launched since it was loaded."""
    return int(lib().gd_kernel_launches())


class GpuError(RuntimeError):
    pass


def _check(rc):
    if rc < 0:
        raise GpuError(lib().gd_last_error().decode())
    return rc


class _BlockRef:
    def __init__(self, blk: dazzdb.Block):
        self.bases = np.ascontiguousarray(blk.bases, dtype=np.uint8)
        self.boff = np.ascontiguousarray(blk.boff, dtype=np.int64)
        self.rlen = np.ascontiguousarray(blk.rlen, dtype=np.int32)
        s = GdBlock()
        s.bases = self.bases.ctypes.data + 1
        s.boff = self.boff.ctypes.data
        s.rlen = self.rlen.ctypes.data
        s.nreads = blk.nreads
        s.maxlen = blk.maxlen
        s.totlen = blk.totlen
        s.ufirst = blk.ufirst
        if blk.mask is not None:
            anno = [0]
            data = []
            for iv in blk.mask:
                for a, b in iv:
                    data += [a, b]
                anno.append(len(data))
            self.anno = np.array(anno, dtype=np.int64)
            self.data = np.array(data + [0], dtype=np.int32)
            s.mask_anno = self.anno.ctypes.data
            s.mask_data = self.data.ctypes.data
        self.s = s


class Context:
    """One GPU context of the overlap path (the current CUDA device)."""

    def __init__(self):
        L = lib()
        self.h = L.gd_create()
        if not self.h:
            raise GpuError(L.gd_last_error().decode())
        self.tspace = 100
        self._nreads = {}

    def close(self):
        if self.h:
            lib().gd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_filter_params(self, kmer=14, binshift=6, suppress=0, hitmin=35):
        _check(lib().gd_set_filter_params(self.h, kmer, binshift, suppress, hitmin))

    def new_align_spec(self, ave_corr, trace_space, freq, symmetric=True, only_identity=False, no_trace=False):
        f = (C.c_float * 4)(*[float(x) for x in freq])
        self.tspace = trace_space
        _check(lib().gd_new_align_spec(self.h, ave_corr, trace_space, f, int(symmetric), int(only_identity),
                                       int(no_trace)))

    def set_globals(self, minover=2000, identity=False, mem_limit=0):
        _check(lib().gd_set_globals(self.h, minover, int(identity), int(mem_limit)))

    def load_block(self, slot, blk):
        r = _BlockRef(blk)
        _check(lib().gd_load_block(self.h, slot, C.byref(r.s)))
        self._nreads[slot] = blk.nreads

    def complement_block(self, src, dst):
        _check(lib().gd_complement_block(self.h, src, dst))

    def timer_mark(self, which):
        _check(lib().gd_timer_mark(self.h, which))

    def timer_elapsed_ms(self):
        ms = lib().gd_timer_elapsed_ms(self.h)
        if ms < 0:
            raise GpuError(lib().gd_last_error().decode())
        return ms

    def sort_kmers(self, slot):
        return _check(lib().gd_sort_kmers(self.h, slot))

    def get_kmers(self, slot, n):
        code = np.zeros(max(n, 1), np.uint64)
        read = np.zeros(max(n, 1), np.int32)
        rpos = np.zeros(max(n, 1), np.int32)
        k = _check(lib().gd_get_kmers(self.h, slot, code.ctypes.data, read.ctypes.data, rpos.ctypes.data, n))
        return code[:k], read[:k], rpos[:k]

    def set_biased(self, biased=True):
        """daligner's -b: frequency-weighted tuples in the index (weights from new_align_spec's freq)."""
        _check(lib().gd_set_biased(self.h, int(bool(biased))))

    def set_variant(self, variant, hgap=0):
        """1 = daligner (default), 2 = daligner2 (modimizer seeds; hgap = its -H)."""
        _check(lib().gd_set_variant(self.h, int(variant), int(hgap)))

    def match_filter2(self, bslot, cslot, self_cmp):
        """daligner2's Match_Filter: A against bslot in both orientations (cslot = complemented B)."""
        _check(lib().gd_match_filter2(self.h, bslot, cslot, int(self_cmp)))

    def test_handle_redundancies_d2(self, aseq, bseq, tspace, comp, hdr, traces, novls, has_b, tcap):
        """Test hook: daligner2's Handle_Redundancies of one pair on the device.  aseq/bseq
        carry a 4 before and after the read."""
        L = lib()
        fn = L.gd_test_handle_redundancies_d2
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        aseq = np.ascontiguousarray(aseq, np.uint8)
        bseq = np.ascontiguousarray(bseq, np.uint8)
        hdr = np.ascontiguousarray(hdr, np.int32)
        traces = np.ascontiguousarray(traces, np.uint16)
        oh = np.zeros(max(hdr.size, 6), np.int32)
        ot = np.zeros(max(int(tcap), 1), np.uint16)
        n = _check(fn(self.h, aseq.ctypes.data + 1, bseq.ctypes.data + 1, aseq.size - 2, bseq.size - 2, tspace, comp,
                      novls, int(has_b), hdr.ctypes.data, traces.ctypes.data, oh.ctypes.data, ot.ctypes.data,
                      int(tcap)))
        return n, oh.reshape(-1, 6), ot

    def match_filter(self, bslot, comp, self_cmp):
        _check(lib().gd_match_filter(self.h, bslot, int(comp), int(self_cmp)))

    def get_hits(self):
        n = _check(lib().gd_get_hits(self.h, None, 0))
        rows = np.zeros((max(n, 1), 4), np.int32)
        _check(lib().gd_get_hits(self.h, rows.ctypes.data, n))
        return rows[:n]

    def sort_overlaps(self):
        """Sorts the overlap buffer on the device; returns (records, trace bytes) kept."""
        tb = C.c_int64()
        n = _check(lib().gd_sort_overlaps(self.h, C.byref(tb)))
        return n, tb.value

    def overlaps(self, out=None):
        """The overlap buffer, sorted like the .las file: (records, trace bytes).  out may
        give (records array of OVL_DTYPE, uint8 array) to fill, e.g. views of pinned memory;
        they must be large enough, and the views returned are their prefixes."""
        n, tb = self.sort_overlaps()
        if out is None:
            recs = np.empty(max(n, 1), OVL_DTYPE)
            tr = np.empty(max(tb, 1), np.uint8)
        else:
            recs, tr = out
            if recs.dtype != OVL_DTYPE or recs.size < n or tr.size < tb or not (recs.flags.c_contiguous and
                                                                               tr.flags.c_contiguous):
                raise ValueError(f"output buffers too small or wrong type for {n} records / {tb} trace bytes")
        k = _check(lib().gd_get_overlaps(self.h, recs.ctypes.data, tr.ctypes.data, n, tb))
        assert k == n
        return recs[:k], tr[:tb]

    def write_overlap_buffer(self, run_id, ablock, bblock, last_read):
        _check(lib().gd_write_overlap_buffer(self.h, run_id, ablock.encode(), bblock.encode(), last_read))

    def compute_trace_pts(self, recs, trace, aslot=0, bslot=0, cslot=2):
        """Exact diffs of each record (Compute_Trace_PTS) from the loaded blocks."""
        recs = np.ascontiguousarray(recs, dtype=OVL_DTYPE)
        trace = np.ascontiguousarray(trace, dtype=np.uint8)
        out = np.zeros(max(recs.size, 1), np.int32)
        _check(lib().gd_compute_trace_pts(self.h, aslot, bslot, cslot, recs.ctypes.data, trace.ctypes.data, recs.size,
                                          out.ctypes.data))
        return out[:recs.size]

    def dust(self, slot, freq, window=64, thresh=2.0, mflag=10, biased=False):
        """DBdust of the block in slot: (anno int64[nreads+1] byte offsets, data int32 pairs)."""
        fr = (C.c_float * 4)(*[float(x) for x in freq])
        anno = np.zeros(self._nreads[slot] + 1, np.int64)
        data = np.zeros(1 << 20, np.int32)
        n = _check(lib().gd_dust(self.h, slot, window, thresh, mflag, int(biased), fr, anno.ctypes.data,
                                 data.ctypes.data, data.size))
        if n > data.size:   # larger than the first guess: run again with room for all
            data = np.zeros(n, np.int32)
            _check(lib().gd_dust(self.h, slot, window, thresh, mflag, int(biased), fr, anno.ctypes.data,
                                 data.ctypes.data, n))
        return anno, data[:n]

    def las_sort(self, in_path, out_path):
        """LAsort of one .las file on the device; returns the number of records."""
        return _check(lib().gd_las_sort(self.h, os.fsencode(in_path), os.fsencode(out_path)))

    def set_wave_limit(self, limit):
        """Test hook: the widest band of the main aligner kernel, 128 (default) or 32."""
        _check(lib().gd_set_wave_limit(self.h, int(limit)))

    def set_capacities(self, pebbles=0, traces=0, paths=0, records=0, trace_bytes=0):
        """Test hook: the aligner's starting capacities (0 keeps one); outgrown ones are grown
        and the alignment stage re-run."""
        _check(lib().gd_set_capacities(self.h, int(pebbles), int(traces), int(paths), int(records),
                                       int(trace_bytes)))

    def set_align_schedule(self, edges=(), kinds=None):
        """() = one persistent aligner launch over all pair groups (default); else one launch
        per length class split at these alen + blen edges (bp); kinds (one per class, longest
        first): 0 = the 128-diagonal warp instance, 1 = the 512-diagonal instance, 2 = the duo
        instance (two 16-lane teams per warp, 128-diagonal rings).  With no edges, kinds holds the
        one persistent launch's instance."""
        e = np.ascontiguousarray(edges, np.int32)
        k = None if kinds is None else np.ascontiguousarray(kinds, np.int32)
        if k is not None and k.size != e.size + 1:
            raise ValueError("one instance kind per length class (len(edges) + 1)")
        self._sched = (e, k)   # keep the arrays alive for the call
        _check(lib().gd_set_align_schedule(self.h, int(e.size), e.ctypes.data if e.size else None,
                                           k.ctypes.data if k is not None else None))

    def test_wait_expiry(self, polls):
        """Test hook: the radix sort's bounded mbarrier wait run out on a copy never issued;
        returns (status of the sort's wait check, its error text)."""
        rc = lib().gd_test_wait_expiry(self.h, int(polls))
        return rc, (lib().gd_last_error() or b"").decode()

    def las_merge(self, in_paths, out_path):
        """LAmerge of .las files on the device; returns the number of records."""
        arr = (C.c_char_p * len(in_paths))(*[os.fsencode(p) for p in in_paths])
        return _check(lib().gd_las_merge(self.h, arr, len(in_paths), os.fsencode(out_path)))

    def reset_overlap_buffer(self):
        _check(lib().gd_reset_overlap_buffer(self.h))

    def stats(self):
        st = GdStats()
        _check(lib().gd_get_stats(self.h, C.byref(st)))
        return {k: (list(getattr(st, k)) if hasattr(getattr(st, k), "__len__") else getattr(st, k))
                for k, _ in GdStats._fields_}

    # learned triage of pair groups (marvel_b200.triage drives these)
    def triage_collect(self, on=True):
        _check(lib().gd_triage_collect(self.h, int(bool(on))))

    def triage_groups(self):
        """Collected rows: (features n x 12 float32, records uint32, cells uint32)."""
        n = _check(lib().gd_triage_get_groups(self.h, None, None, None, 0))
        feat = np.zeros((n, TRI_NF), np.float32)
        rec = np.zeros(n, np.uint32)
        cells = np.zeros(n, np.uint32)
        _check(lib().gd_triage_get_groups(self.h, feat.ctypes.data, rec.ctypes.data, cells.ctypes.data, n))
        return feat, rec, cells

    def triage_reset(self):
        _check(lib().gd_triage_reset(self.h))

    def triage_set_model(self, params, threshold=0.0):
        if params is None:
            _check(lib().gd_triage_set_model(self.h, None, 0.0))
            return
        self._tri_params = np.ascontiguousarray(params, np.float32)
        assert self._tri_params.size == TRI_NPARAM
        _check(lib().gd_triage_set_model(self.h, self._tri_params.ctypes.data, float(threshold)))

    def mlp_forward(self, params, feat):
        params = np.ascontiguousarray(params, np.float32)
        feat = np.ascontiguousarray(feat, np.float32).reshape(-1, TRI_NF)
        prob = np.zeros(feat.shape[0], np.float32)
        _check(lib().gd_mlp_forward(self.h, params.ctypes.data, feat.ctypes.data, feat.shape[0], prob.ctypes.data))
        return prob

    def mlp_grad(self, params, feat, label, pos_weight=1.0):
        params = np.ascontiguousarray(params, np.float32)
        feat = np.ascontiguousarray(feat, np.float32).reshape(-1, TRI_NF)
        label = np.ascontiguousarray(label, np.float32)
        grad = np.zeros(TRI_NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        _check(lib().gd_mlp_grad(self.h, params.ctypes.data, feat.ctypes.data, label.ctypes.data, feat.shape[0],
                                 float(pos_weight), grad.ctypes.data, loss.ctypes.data))
        return grad, float(loss[0])

    def mlp_train(self, feat, label, params, epochs=20, batch=4096, lr=2e-3, pos_weight=1.0, seed=1):
        feat = np.ascontiguousarray(feat, np.float32).reshape(-1, TRI_NF)
        label = np.ascontiguousarray(label, np.float32)
        out = np.array(params, np.float32, copy=True)
        losses = np.zeros(epochs, np.float32)
        _check(lib().gd_mlp_train(self.h, feat.ctypes.data, label.ctypes.data, feat.shape[0], int(epochs), int(batch),
                                  float(lr), float(pos_weight), int(seed), out.ctypes.data, losses.ctypes.data))
        return out, losses

    def local_alignment_batch(self, abases, aoff, alen, bbases, boff, blen, diag, anti, comp, trstride=None):
        n = len(diag)
        if trstride is None:
            trstride = 2 * (4 * (int(max(np.max(alen), np.max(blen))) // self.tspace + 2) + 16)
        out = np.zeros((n, 12), np.int32)
        tr = np.zeros((n, trstride), np.uint16)
        cells = np.zeros(n, np.int64)
        abases = np.ascontiguousarray(abases, np.uint8)
        bbases = np.ascontiguousarray(bbases, np.uint8)
        arrs = [np.ascontiguousarray(x, t) for x, t in ((aoff, np.int64), (alen, np.int32), (boff, np.int64),
                                                         (blen, np.int32), (diag, np.int32), (anti, np.int32))]
        _check(lib().gd_local_alignment_batch(self.h, abases.ctypes.data, abases.size, bbases.ctypes.data,
                                              bbases.size, *[a.ctypes.data for a in arrs], n, int(comp),
                                              out.ctypes.data, tr.ctypes.data, trstride, cells.ctypes.data))
        return out, tr, cells


def daligner_block(ctx: Context, A: dazzdb.Block, B: dazzdb.Block | None = None, *, k=14, w=6, h=35, t=0, e=0.70,
                   l=1000, s=100, M=32, symmetric=True, identity=False, only_identity=False, no_trace=False):
    """One daligner block comparison on the GPU (dalign/daligner.c:957-1014): A against B
    (or against itself when B is None) in both orientations.  Returns the overlap buffer
    as (records, trace bytes), sorted like the .las file."""
    self_cmp = B is None
    ctx.set_filter_params(k, w, t, h)
    ctx.new_align_spec(e, s, A.freq, symmetric and True, only_identity, no_trace)
    ctx.set_globals(2 * l, identity or only_identity, int(M) * 0x40000000)
    ctx.reset_overlap_buffer()
    ctx.load_block(0, A)
    if not self_cmp:
        ctx.load_block(1, B)
    run_loaded(ctx, self_cmp)
    return ctx.overlaps()


def run_loaded(ctx: Context, self_cmp: bool):
    """The per-block device pipeline once the blocks are resident: Sort_Kmers(A),
    Match_Filter(A, B), complement_DB(B), Sort_Kmers(cB), Match_Filter(A, cB)
    (dalign/daligner.c:957-1012)."""
    ctx.sort_kmers(0)
    if self_cmp:
        ctx.match_filter(0, 0, 1)
        ctx.complement_block(0, 2)
    else:
        ctx.sort_kmers(1)
        ctx.match_filter(1, 0, 0)
        ctx.complement_block(1, 2)
    ctx.sort_kmers(2)
    ctx.match_filter(2, 1, int(self_cmp))


def daligner2_block(ctx: Context, A: dazzdb.Block, B: dazzdb.Block | None = None, *, k=14, w=6, h=35, t=0,
                    e=0.70, l=1000, s=100, M=32, H=0, symmetric=True, identity=False):
    """One daligner2 block comparison on the GPU (dalign2/daligner.c:654-790): A against B (or
    against itself when B is None), both orientations from one join.  Returns the overlap
    buffer as (records, trace bytes), sorted like the .las file."""
    self_cmp = B is None
    ctx.set_variant(2, H)
    ctx.set_filter_params(k, w, t, h)
    ctx.new_align_spec(e, s, A.freq, symmetric, False, False)
    ctx.set_globals(2 * l, identity, int(M) * 0x40000000)
    ctx.reset_overlap_buffer()
    ctx.load_block(0, A)
    if not self_cmp:
        ctx.load_block(1, B)
    run_loaded2(ctx, self_cmp)
    return ctx.overlaps()


def run_loaded2(ctx: Context, self_cmp: bool):
    """daligner2's per-block device pipeline once the blocks are resident (context in variant
    2): Sort_Kmers(A), Sort_Kmers(B), the complemented B block for the complement pairs'
    alignments (CopyAndComp per pair in the reference), Match_Filter(A, B)."""
    ctx.sort_kmers(0)
    if self_cmp:
        ctx.complement_block(0, 2)
        ctx.match_filter2(0, 2, 1)
    else:
        ctx.sort_kmers(1)
        ctx.complement_block(1, 2)
        ctx.match_filter2(1, 2, 0)


def write_las(path, recs, trace, tspace):
    """Writes records (OVL_DTYPE, already sorted) and their trace bytes as a .las file."""
    tb = 1 if tspace <= 125 else 2
    with open(path, "wb") as f:
        f.write(np.int64(recs.size).tobytes())
        f.write(np.int32(tspace).tobytes())
        for r in recs:
            f.write(np.array([r["tlen"], r["diffs"], r["abpos"], r["bbpos"], r["aepos"], r["bepos"]], "<i4").tobytes())
            f.write(np.uint32(r["flags"]).tobytes())
            f.write(np.array([r["aread"], r["bread"], 0], "<i4").tobytes())
            o = int(r["toff"])
            f.write(trace[o:o + int(r["tlen"]) * tb].tobytes())

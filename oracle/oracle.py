"""ctypes binding of the CPU restatement (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, by the smoke check and by bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


class or_block(C.Structure):
    _fields_ = [("bases", C.c_void_p), ("boff", C.c_void_p), ("rlen", C.c_void_p), ("nreads", C.c_int32),
                ("maxlen", C.c_int32), ("totlen", C.c_int64), ("ufirst", C.c_int32),
                ("mask_anno", C.c_void_p), ("mask_data", C.c_void_p)]


class or_params(C.Structure):
    _fields_ = [("kmer", C.c_int32), ("binshift", C.c_int32), ("suppress", C.c_int32), ("hitmin", C.c_int32),
                ("ave_corr", C.c_double), ("tspace", C.c_int32), ("minover", C.c_int32),
                ("symmetric", C.c_int32), ("identity", C.c_int32), ("only_identity", C.c_int32),
                ("no_trace", C.c_int32), ("mem_limit", C.c_uint64), ("freq", C.c_float * 4),
                ("hgap", C.c_int32), ("variant", C.c_int32), ("biased", C.c_int32)]


class or_overlap(C.Structure):
    _fields_ = [("tlen", C.c_int32), ("diffs", C.c_int32), ("abpos", C.c_int32), ("bbpos", C.c_int32),
                ("aepos", C.c_int32), ("bepos", C.c_int32), ("flags", C.c_uint32), ("aread", C.c_int32),
                ("bread", C.c_int32), ("toff", C.c_int64)]


class or_result(C.Structure):
    _fields_ = [("novl", C.c_int64), ("ovl", C.POINTER(or_overlap)), ("trace", C.POINTER(C.c_uint8)),
                ("tbytes_total", C.c_int64), ("tbytes", C.c_int32),
                ("kmers_a", C.c_int64), ("kmers_b", C.c_int64), ("hits_n", C.c_int64), ("hits_c", C.c_int64),
                ("seeds_n", C.c_int64), ("seeds_c", C.c_int64), ("cells", C.c_int64), ("snake_steps", C.c_int64),
                ("status", C.c_int32)]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle liboracle.so)")
        _lib = C.CDLL(path)
        _lib.or_daligner.argtypes = [C.POINTER(or_block)] * 3 + [C.POINTER(or_params), C.c_int, C.POINTER(or_result)]
        _lib.or_daligner2.argtypes = [C.POINTER(or_block)] * 3 + [C.POINTER(or_params), C.c_int, C.POINTER(or_result)]
        _lib.or_free_result.argtypes = [C.POINTER(or_result)]
        _lib.or_sort_kmers2.argtypes = [C.POINTER(or_block), C.POINTER(or_params), C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_sort_kmers2.restype = C.c_int64
        _lib.or_sort_kmers.argtypes = [C.POINTER(or_block), C.POINTER(or_params), C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.or_sort_kmers.restype = C.c_int64
        _lib.or_match_hits.argtypes = [C.POINTER(or_block), C.POINTER(or_block), C.POINTER(or_params), C.c_int,
                                       C.POINTER(C.c_void_p), C.POINTER(C.c_int32)]
        _lib.or_match_hits.restype = C.c_int64
        _lib.or_local_alignment.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.POINTER(or_params), C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.POINTER(C.c_int64)]
        _lib.or_free.argtypes = [C.c_void_p]
        _lib.or_trace_pts_diffs.argtypes = [C.c_void_p] * 2 + [C.c_int] * 6 + [C.c_void_p, C.c_void_p, C.c_int,
                                                                                C.c_int, C.POINTER(C.c_int32)]
    return _lib


class BlockRef:
    """Keeps the numpy arrays alive behind an or_block."""

    def __init__(self, blk):
        self.blk = blk
        self.bases = np.ascontiguousarray(blk.bases)
        self.boff = np.ascontiguousarray(blk.boff, dtype=np.int64)
        self.rlen = np.ascontiguousarray(blk.rlen, dtype=np.int32)
        s = or_block()
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
        else:
            s.mask_anno = None
            s.mask_data = None
        self.s = s


def make_params(freq, k=14, w=6, h=35, t=0, e=0.70, l=1000, s=100, M=32, symmetric=True, identity=False,
                only_identity=False, no_trace=False, H=0, variant=1, biased=False):
    """variant 1 = daligner (dalign/), 2 = daligner2 (dalign2/, where -H is live); biased = daligner's -b."""
    p = or_params()
    p.hgap = int(H)
    p.variant = int(variant)
    p.biased = int(biased)
    p.kmer, p.binshift, p.suppress, p.hitmin = k, w, t, h
    p.ave_corr = e
    p.tspace = s
    p.minover = 2 * l
    p.symmetric = int(symmetric)
    p.identity = int(identity or only_identity)
    p.only_identity = int(only_identity)
    p.no_trace = int(no_trace)
    p.mem_limit = int(M) * 0x40000000
    for i in range(4):
        p.freq[i] = float(freq[i])
    return p


def daligner(a, b, bc, params, self_cmp):
    """Run the restated overlap path; returns (records list of dicts-as-tuples, traces, stats)."""
    L = lib()
    fn = L.or_daligner2 if params.variant == 2 else L.or_daligner
    ra, rb, rc = BlockRef(a), BlockRef(b), BlockRef(bc)
    res = or_result()
    fn(C.byref(ra.s), C.byref(rb.s), C.byref(rc.s), C.byref(params), int(self_cmp), C.byref(res))
    n = res.novl
    tb = res.tbytes
    recs = []
    traces = []
    if n:
        arr = np.ctypeslib.as_array(C.cast(res.ovl, C.POINTER(C.c_uint8)), shape=(n * C.sizeof(or_overlap),))
        ov = np.frombuffer(arr.tobytes(), dtype=np.dtype([("tlen", "<i4"), ("diffs", "<i4"), ("abpos", "<i4"),
                                                          ("bbpos", "<i4"), ("aepos", "<i4"), ("bepos", "<i4"),
                                                          ("flags", "<u4"), ("aread", "<i4"), ("bread", "<i4"),
                                                          ("_pad", "<i4"), ("toff", "<i8")]))
        tr = np.ctypeslib.as_array(res.trace, shape=(max(res.tbytes_total, 1),)).copy()
        recs = ov.copy()
        for i in range(n):
            o = int(ov["toff"][i])
            L_ = int(ov["tlen"][i]) * tb
            traces.append(tr[o:o + L_].view("<u1" if tb == 1 else "<u2").copy())
    stats = {k: getattr(res, k) for k in ("kmers_a", "kmers_b", "hits_n", "hits_c", "seeds_n", "seeds_c", "cells",
                                          "status")}
    L.or_free_result(C.byref(res))
    return recs, traces, stats


def write_las(path, recs, traces, tspace):
    tb = 1 if tspace <= 125 else 2
    with open(path, "wb") as f:
        f.write(np.int64(len(traces)).tobytes())
        f.write(np.int32(tspace).tobytes())
        for i in range(len(traces)):
            r = recs[i]
            f.write(np.array([r["tlen"], r["diffs"], r["abpos"], r["bbpos"], r["aepos"], r["bepos"]],
                             dtype="<i4").tobytes())
            f.write(np.uint32(r["flags"]).tobytes())
            f.write(np.array([r["aread"], r["bread"], 0], dtype="<i4").tobytes())
            f.write(traces[i].astype("<u1" if tb == 1 else "<u2").tobytes())


def sort_kmers(blk, params):
    L = lib()
    r = BlockRef(blk)
    n = blk.totlen + 1
    code = np.zeros(n, np.uint64)
    read = np.zeros(n, np.int32)
    rpos = np.zeros(n, np.int32)
    k = L.or_sort_kmers(C.byref(r.s), C.byref(params), code.ctypes.data, read.ctypes.data, rpos.ctypes.data)
    return code[:k], read[:k], rpos[:k]


def sort_kmers2(blk, params):
    """daligner2's sorted modimizer index: (code, (read << 1) | strand, rpos)."""
    L = lib()
    r = BlockRef(blk)
    n = 2 * blk.totlen + 2
    code = np.zeros(n, np.uint64)
    read = np.zeros(n, np.int32)
    rpos = np.zeros(n, np.int32)
    k = L.or_sort_kmers2(C.byref(r.s), C.byref(params), code.ctypes.data, read.ctypes.data, rpos.ctypes.data)
    return code[:k], read[:k], rpos[:k]


def match_hits(a, b, params, self_cmp):
    L = lib()
    ra, rb = BlockRef(a), BlockRef(b)
    ptr = C.c_void_p()
    lim = C.c_int32()
    n = L.or_match_hits(C.byref(ra.s), C.byref(rb.s), C.byref(params), int(self_cmp), C.byref(ptr), C.byref(lim))
    arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(max(n, 1) * 4,)).reshape(-1, 4)[:n].copy()
    L.or_free(ptr)
    return arr, lim.value   # columns: diag, apos, aread, bread


def local_alignment(aseq, bseq, comp, diag, anti, params):
    """aseq/bseq: uint8 arrays with a 4 before and after the read."""
    L = lib()
    aseq = np.ascontiguousarray(aseq, np.uint8)
    bseq = np.ascontiguousarray(bseq, np.uint8)
    alen, blen = aseq.size - 2, bseq.size - 2
    cap = 4 * (max(alen, blen) // params.tspace + 2) + 16
    out = np.zeros(12, np.int32)
    at = np.zeros(cap, np.uint16)
    bt = np.zeros(cap, np.uint16)
    cells = C.c_int64()
    L.or_local_alignment(aseq.ctypes.data + 1, bseq.ctypes.data + 1, alen, blen, comp, diag, anti, C.byref(params),
                         out.ctypes.data, at.ctypes.data, bt.ctypes.data, C.byref(cells))
    return out, at[:out[5]].copy(), bt[:out[11]].copy(), cells.value


def trace_pts_diffs(aread_seq, bread_seq, rec, trace, tspace):
    """Compute_Trace_PTS diffs of one record; sequences are the reads' bases (B complemented
    for a COMP record), trace the record's trace values."""
    L = lib()
    a = np.ascontiguousarray(aread_seq, np.uint8)
    b = np.ascontiguousarray(bread_seq, np.uint8)
    out = C.c_int32()
    t8 = np.ascontiguousarray(trace, np.uint8) if tspace <= 125 else None
    t16 = None if tspace <= 125 else np.ascontiguousarray(trace, np.uint16)
    L.or_trace_pts_diffs(a.ctypes.data, b.ctypes.data, a.size, b.size, int(rec["abpos"]), int(rec["bbpos"]),
                         int(rec["aepos"]), int(rec["bepos"]), None if t8 is None else t8.ctypes.data,
                         None if t16 is None else t16.ctypes.data, int(rec["tlen"]), tspace, C.byref(out))
    return out.value


def dust(block, window=64, thresh=2.0, mflag=10, biased=False):
    """DBdust's scan of every read of a block (dust_oracle.c): (anno int64[n+1] byte offsets,
    data int32 pairs), the .dust.anno / .dust.data layout."""
    fn = lib().or_dust_read
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    f = [np.float32(x) for x in block.freq]
    skew = np.zeros(64, np.float64)
    p = 0
    for a in range(4):
        for b in range(4):
            for c in range(4):
                q = np.float32(f[a] * f[b])
                q = np.float32(q * f[c])
                skew[p] = .015625 / float(q)
                p += 1
    n = block.nreads
    anno = np.zeros(n + 1, np.int64)
    out = []
    o = 0
    for r in range(n):
        seq = np.ascontiguousarray(block.read(r), np.uint8)
        L_ = seq.size
        buf = np.zeros(L_ + 8, np.int32)
        work = np.zeros(L_ + 8, np.int32)
        k = fn(seq.ctypes.data, L_, window, thresh, mflag - 1, int(biased), skew.ctypes.data, buf.ctypes.data,
               work.ctypes.data)
        if k < 0:
            raise RuntimeError(f"or_dust_read failed on read {r} ({k})")
        anno[r] = 4 * o
        out.append(buf[:k].copy())
        o += k
    anno[n] = 4 * o
    return anno, (np.concatenate(out) if out else np.zeros(0, np.int32))

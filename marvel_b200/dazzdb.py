"""Dazzler DB and .las file formats (reader and writer), in numpy.

On-disk layout, as the reference defines it:
  * ``X.db``    text stub: files / blocks / size / block boundaries (db/DB.h:239-249)
  * ``.X.idx``  raw ``HITS_DB`` header (88 bytes) + ``HITS_READ[ureads]`` (32 bytes each)
                (db/DB.c:424-450, db/DB.h:163-236)
  * ``.X.bps``  2-bit packed bases, 4 per byte, first base in the high bits
                (db/DB.c:261-309, Compress_Read / Uncompress_Read)
  * ``.las``    ``int64 novl, int32 tspace`` then per overlap a 40-byte record
                ``tlen, diffs, abpos, bbpos, aepos, bepos, flags, aread, bread, pad``
                followed by ``tlen`` trace bytes (1 byte when tspace <= 125, else 2)
                (dalign/align.c:3325-3350, dalign/align.h:307-321)

``Block`` holds a loaded block the way daligner keeps it in memory
(db/DB.c:1349-1410, Read_All_Sequences): one byte per base (0..3), a 4 before the first
read and after every read, and ``boff[i]`` the offset of read i in that buffer.
"""
from __future__ import annotations

import dataclasses
import os
import numpy as np

HITS_DB_SIZE = 88
HITS_READ_DTYPE = np.dtype([("rlen", "<i4"), ("_p0", "<i4"), ("boff", "<i8"),
                            ("coff", "<i8"), ("flags", "<i4"), ("_p1", "<i4")])
assert HITS_READ_DTYPE.itemsize == 32
DB_BEST = 0x0800

LAS_REC_DTYPE = np.dtype([("tlen", "<i4"), ("diffs", "<i4"), ("abpos", "<i4"), ("bbpos", "<i4"),
                          ("aepos", "<i4"), ("bepos", "<i4"), ("flags", "<u4"), ("aread", "<i4"),
                          ("bread", "<i4"), ("pad", "<i4")])
assert LAS_REC_DTYPE.itemsize == 40


def _split_path(path):
    d, base = os.path.split(path)
    if base.endswith(".db"):
        base = base[:-3]
    part = 0
    root = base
    if "." in base:
        stem, suf = base.rsplit(".", 1)
        if suf.isdigit() and int(suf) > 0:
            root, part = stem, int(suf)
    return d or ".", root, part


@dataclasses.dataclass
class Block:
    bases: np.ndarray      # uint8, [4, read0..., 4, read1..., 4, ...]; bases[boff[i]+1] is read i's first base
    boff: np.ndarray       # int64[nreads+1] offsets *within bases[1:]* (reference convention)
    rlen: np.ndarray       # int32[nreads]
    ufirst: int
    part: int
    freq: np.ndarray       # float32[4]
    maxlen: int
    totlen: int
    root: str = ""
    mask: list | None = None   # per read list of (beg, end) masked intervals, or None

    @property
    def nreads(self):
        return int(self.rlen.size)

    def read(self, i):
        o = int(self.boff[i]) + 1
        return self.bases[o:o + int(self.rlen[i])]


def read_stub(path):
    d, root, part = _split_path(path)
    with open(os.path.join(d, root + ".db")) as f:
        lines = f.read().split("\n")
    nfiles = int(lines[0].split("=")[1])
    i = 1 + nfiles
    blocks = []
    size = None
    if i < len(lines) and lines[i].startswith("blocks"):
        nblocks = int(lines[i].split("=")[1])
        size = int(lines[i + 1].split("=")[1])
        blocks = [int(x) for x in lines[i + 2:i + 3 + nblocks]]
    return d, root, part, blocks, size


def open_block(path) -> Block:
    """Load a DB (or one block ``X.n``) like Open_DB_Block + Read_All_Sequences."""
    d, root, part, blocks, _ = read_stub(path)
    with open(os.path.join(d, "." + root + ".idx"), "rb") as f:
        hdr = f.read(HITS_DB_SIZE)
        recs = np.frombuffer(f.read(), dtype=HITS_READ_DTYPE)
    ureads = int(np.frombuffer(hdr[0:4], "<i4")[0])
    freq = np.frombuffer(hdr[4:20], "<f4").copy()
    maxlen = int(np.frombuffer(hdr[20:24], "<i4")[0])
    totlen = int(np.frombuffer(hdr[24:32], "<i8")[0])
    if part > 0:
        ufirst, ulast = blocks[part - 1], blocks[part]
    else:
        ufirst, ulast = 0, ureads
    sub = recs[ufirst:ulast]
    rlen = sub["rlen"].astype(np.int32)
    if part > 0:
        maxlen = int(rlen.max()) if rlen.size else 0
        totlen = int(rlen.sum())
    raw = np.fromfile(os.path.join(d, "." + root + ".bps"), dtype=np.uint8)
    bases, boff = _unpack(raw, sub["boff"], rlen)
    return Block(bases, boff, rlen, ufirst, part, freq, maxlen, totlen, os.path.join(d, root))


def _unpack(raw, foff, rlen):
    n = rlen.size
    boff = np.zeros(n + 1, dtype=np.int64)
    boff[1:] = np.cumsum(rlen.astype(np.int64) + 1)
    out = np.full(int(boff[-1]) + 1 + 4, 4, dtype=np.uint8)
    # unpack everything once, then gather
    q = np.empty(raw.size * 4, dtype=np.uint8)
    q[0::4] = (raw >> 6) & 3
    q[1::4] = (raw >> 4) & 3
    q[2::4] = (raw >> 2) & 3
    q[3::4] = raw & 3
    for i in range(n):
        L = int(rlen[i])
        s = int(foff[i]) * 4
        o = int(boff[i]) + 1
        out[o:o + L] = q[s:s + L]
    return out, boff


def load_track(b: Block, name: str):
    """Adds interval track `name` as b.mask (the .anno/.data layout Load_Track reads,
    db/DB.c:967-1120; a per-block ".X.n.track" file wins over the whole-DB one).  A second
    track is united with the masks already there."""
    d, root = os.path.split(b.root)
    cands = []
    if b.part > 0:
        cands.append((os.path.join(d, f".{root}.{b.part}.{name}"), True))
    cands.append((os.path.join(d, f".{root}.{name}"), False))
    for base, ispart in cands:
        if os.path.exists(base + ".anno"):
            break
    else:
        raise FileNotFoundError(f"track {name} not found for {b.root}")
    raw = open(base + ".anno", "rb").read()
    tracklen, size = np.frombuffer(raw[:8], "<i4")
    anno = np.frombuffer(raw[8:], "<i8" if size == 8 else "<i4").astype(np.int64)
    first = 0 if ispart else b.ufirst
    anno = anno[first:first + b.nreads + 1]
    data = np.fromfile(base + ".data", dtype="<i4")
    off = int(anno[0]) // 4
    iv = []
    for i in range(b.nreads):
        s, e = int(anno[i]) // 4, int(anno[i + 1]) // 4
        x = data[s:e]
        iv.append([(int(x[j]), int(x[j + 1])) for j in range(0, len(x), 2)])
    del off
    if b.mask is None:
        b.mask = iv
    else:
        merged = []
        for a, c in zip(b.mask, iv):
            allv = sorted(a + c)
            out = []
            for s, e in allv:
                if out and s <= out[-1][1]:
                    out[-1] = (out[-1][0], max(out[-1][1], e))
                else:
                    out.append((s, e))
            merged.append(out)
        b.mask = merged
    return b


def complement_block(b: Block) -> Block:
    """Reverse-complement every read in place of a copy (dalign/daligner.c:474-573)."""
    bases = b.bases.copy()
    for i in range(b.nreads):
        o = int(b.boff[i]) + 1
        L = int(b.rlen[i])
        bases[o:o + L] = 3 - b.bases[o:o + L][::-1]
    freq = b.freq[[3, 2, 1, 0]].copy()
    mask = None
    if b.mask is not None:
        mask = [[(int(b.rlen[i]) - e, int(b.rlen[i]) - s) for (s, e) in reversed(iv)] for i, iv in enumerate(b.mask)]
    return dataclasses.replace(b, bases=bases, freq=freq, mask=mask)


def write_db(path_root, reads, block_mbp=200, ufirst_split=True):
    """Write ``root.db``/``.root.idx``/``.root.bps`` for a list of uint8 reads (0..3).

    The result loads the same way as an FA2db + DBsplit -s<block_mbp> database: same read
    order, same 2-bit packing, same block boundaries (db/DBsplit.c:207-246)."""
    d, root = os.path.split(path_root)
    d = d or "."
    n = len(reads)
    rlen = np.array([r.size for r in reads], dtype=np.int64)
    clen = (rlen + 3) // 4
    foff = np.zeros(n, dtype=np.int64)
    foff[1:] = np.cumsum(clen)[:-1]
    allb = np.concatenate(reads) if n else np.zeros(0, np.uint8)
    with open(os.path.join(d, "." + root + ".bps"), "wb") as f:
        for r in reads:
            pad = (-r.size) % 4
            x = np.concatenate([r, np.zeros(pad, np.uint8)]).reshape(-1, 4)
            f.write(((x[:, 0] << 6) | (x[:, 1] << 4) | (x[:, 2] << 2) | x[:, 3]).astype(np.uint8).tobytes())
    counts = np.bincount(allb, minlength=4).astype(np.float64)
    totlen = int(rlen.sum())
    freq = (counts / max(totlen, 1)).astype(np.float32)
    hdr = bytearray(HITS_DB_SIZE)
    hdr[0:4] = np.int32(n).tobytes()
    hdr[4:20] = freq.tobytes()
    hdr[20:24] = np.int32(int(rlen.max()) if n else 0).tobytes()
    hdr[24:32] = np.int64(totlen).tobytes()
    recs = np.zeros(n, dtype=HITS_READ_DTYPE)
    recs["rlen"] = rlen
    recs["boff"] = foff
    recs["coff"] = -1
    recs["flags"] = DB_BEST
    with open(os.path.join(d, "." + root + ".idx"), "wb") as f:
        f.write(bytes(hdr))
        f.write(recs.tobytes())
    # block boundaries exactly as DBsplit -s computes them
    size = int(block_mbp * 1000000)
    bounds = [0]
    tot = 0
    for i in range(n):
        tot += int(rlen[i])
        if tot >= size:
            bounds.append(i + 1)
            tot = 0
    if bounds[-1] != n:
        bounds.append(n)
    with open(os.path.join(d, root + ".db"), "w") as f:
        f.write("files = %9d\n" % 1)
        f.write("  %9d %s %s\n" % (n, root, "sim"))
        f.write("blocks = %9d\n" % (len(bounds) - 1))
        f.write("size = %9d\n" % block_mbp)
        for b in bounds:
            f.write(" %9d\n" % b)
    return len(bounds) - 1


def read_las(path):
    """Returns (tspace, records structured array, list of trace arrays)."""
    with open(path, "rb") as f:
        data = f.read()
    novl = int(np.frombuffer(data[0:8], "<i8")[0])
    tspace = int(np.frombuffer(data[8:12], "<i4")[0])
    tbytes = 1 if tspace <= 125 else 2
    recs = np.zeros(novl, dtype=LAS_REC_DTYPE)
    traces = []
    off = 12
    for i in range(novl):
        r = np.frombuffer(data, LAS_REC_DTYPE, 1, off)[0]
        recs[i] = r
        off += 40
        tl = int(r["tlen"])
        t = np.frombuffer(data, "<u1" if tbytes == 1 else "<u2", tl, off).copy()
        traces.append(t)
        off += tl * tbytes
    assert off == len(data), (off, len(data))
    return tspace, recs, traces


def las_equal(path_a, path_b, key="overlap", pad=False):
    """Record-level comparison of two .las files that accepts any order among records whose
    sort keys tie: (aread, bread, COMP, abpos) for key="overlap" (Write_Overlap_Buffer,
    dalign/align.c:5786-5813), (aread, bread, abpos) for key="lasort" (dalign/LAsort.c:65-90).
    The 4 pad bytes of each record (uninitialised in daligner's output) are ignored unless
    pad=True.  Returns (equal, message)."""
    ta, ra, xa = read_las(path_a)
    tb, rb, xb = read_las(path_b)
    if ta != tb:
        return False, f"tspace {ta} != {tb}"
    if ra.size != rb.size:
        return False, f"novl {ra.size} != {rb.size}"
    fields = [f for f in LAS_REC_DTYPE.names if pad or f != "pad"]

    def canon(recs, traces):
        keys = []
        for i in range(recs.size):
            r = recs[i]
            keys.append(tuple(int(r[f]) for f in fields) + (traces[i].tobytes(),))
        return keys

    ka, kb = canon(ra, xa), canon(rb, xb)
    if ka == kb:
        return True, "identical"
    if sorted(ka) == sorted(kb):
        # same multiset: allowed only if differences are among tied sort keys
        ia, ib, fl, ab = (fields.index(f) for f in ("aread", "bread", "flags", "abpos"))

        def sk(k):
            return (k[ia], k[ib], k[fl] & 1, k[ab]) if key == "overlap" else (k[ia], k[ib], k[ab])
        for x, y in zip(ka, kb):
            if sk(x) != sk(y):
                return False, "same records, different order"
        return True, "identical up to tied sort keys"
    sa, sb = set(ka), set(kb)
    onlya = [k for k in ka if k not in sb]
    onlyb = [k for k in kb if k not in sa]
    return False, f"{len(onlya)} records only in {path_a}, {len(onlyb)} only in {path_b}; first: {onlya[:1]} vs {onlyb[:1]}"


def read_las_arrays(path):
    """Like read_las, as flat arrays for large files: (tspace, records of LAS_REC_DTYPE,
    trace bytes as stored, byte offset of each record's trace in them)."""
    with open(path, "rb") as f:
        data = f.read()
    novl = int(np.frombuffer(data[0:8], "<i8")[0])
    tspace = int(np.frombuffer(data[8:12], "<i4")[0])
    tbytes = 1 if tspace <= 125 else 2
    offs = np.empty(novl, np.int64)
    off = 12
    from_bytes = int.from_bytes
    for i in range(novl):
        offs[i] = off
        off += 40 + from_bytes(data[off:off + 4], "little", signed=True) * tbytes
    assert off == len(data), (off, len(data))
    raw = np.frombuffer(data, np.uint8)
    recs = raw[offs[:, None] + np.arange(40)].copy().view(LAS_REC_DTYPE).reshape(novl)
    nb = recs["tlen"].astype(np.int64) * tbytes
    toff = np.zeros(novl, np.int64)
    if novl:
        toff[1:] = np.cumsum(nb)[:-1]
    idx = np.repeat(offs + 40 - toff, nb) + np.arange(int(nb.sum()), dtype=np.int64)
    return tspace, recs, raw[idx].copy(), toff


def las_digest(recs, trace_bytes, toff, tbytes=1):
    """Order-free SHA-256 of an overlap set: every record's nine fields (tlen, diffs, abpos,
    bbpos, aepos, bepos, flags, aread, bread -- the pad word is left out, it is uninitialised
    in daligner's files) and its trace bytes, over the records sorted by all of them.  Two
    .las files (or a file and an in-memory buffer) have equal digests exactly when they hold
    the same records, whatever the order among tied sort keys.  recs: any structured array
    with those fields; toff: each record's byte offset into trace_bytes.  Returns
    (hex digest, record count)."""
    import hashlib
    names = ("tlen", "diffs", "abpos", "bbpos", "aepos", "bepos", "flags", "aread", "bread")
    n = int(recs.size)
    fixed = np.empty((n, 9), np.int64)
    for j, f in enumerate(names):
        fixed[:, j] = recs[f]
    # primary key first: aread, bread, flags, abpos, aepos, bbpos, bepos, diffs, tlen
    keyorder = (7, 8, 6, 2, 4, 3, 5, 1, 0)
    order = np.lexsort(tuple(fixed[:, j] for j in reversed(keyorder)))
    fixed = fixed[order]
    toff = np.asarray(toff, np.int64)[order]
    nb = fixed[:, 0] * tbytes
    tb = np.asarray(trace_bytes, np.uint8)

    def trace_of(i):
        return tb[toff[i]:toff[i] + nb[i]].tobytes()
    # records whose nine fields all tie are ordered by their trace bytes
    if n > 1:
        same = np.all(fixed[1:] == fixed[:-1], axis=1)
        i = 0
        tied = np.nonzero(same)[0]
        while i < tied.size:
            j = i
            while j + 1 < tied.size and tied[j + 1] == tied[j] + 1:
                j += 1
            lo, hi = int(tied[i]), int(tied[j]) + 2
            sub = sorted(range(lo, hi), key=trace_of)
            order_sub = np.asarray(sub, np.int64)
            toff[lo:hi] = toff[order_sub]
            i = j + 1
    h = hashlib.sha256()
    h.update(fixed.astype("<i4").tobytes())
    ends = np.cumsum(nb)
    idx = np.repeat(toff - (ends - nb), nb) + np.arange(int(nb.sum()), dtype=np.int64)
    h.update(tb[idx].tobytes())
    return h.hexdigest(), n


def las_file_digest(path):
    """las_digest of a .las file: (tspace, hex digest, record count)."""
    tspace, recs, tb, toff = read_las_arrays(path)
    d, n = las_digest(recs, tb, toff, 1 if tspace <= 125 else 2)
    return tspace, d, n

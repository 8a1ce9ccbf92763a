"""Drives one daligner invocation (flags + blocks, dalign/daligner.c:615-1029) through either
the oracle (CPU restatement) or the GPU library, writing .las files with the reference's
directory and file naming (Write_Overlap_Buffer, dalign/align.c:5855-6043)."""
from __future__ import annotations

import os

import numpy as np

from marvel_b200 import dazzdb


def parse_flags(flags):
    o = dict(k=14, w=6, h=35, t=0, e=0.70, l=1000, s=100, M=None, A=False, I=False, O=False, T=False, r=1, m=[],
             H=0, b=False)
    for f in flags:
        c, v = f[1], f[2:]
        if c in "kwhtlsHr":
            o[c] = int(v)
        elif c == "M":
            o["M"] = int(v)
        elif c == "e":
            o["e"] = float(v)
        elif c == "m":
            o["m"].append(v)
        elif c in "AIOTb":
            o[c] = True
        elif c == "j":
            pass
        else:
            raise ValueError(f"unsupported flag {f}")
    return o


def las_names(aname, bname, run_id, symmetric):
    """Paths (relative to the DB directory) Write_Overlap_Buffer writes, in (first, second) order."""
    def split(n):
        root, _, b = n.rpartition(".")
        return root, int(b)
    ar, ai = split(aname)
    br, bi = split(bname)
    d1 = "%03d_%05d" % (run_id, ai)
    d2 = "%03d_%05d" % (run_id, bi)
    if aname == bname or not symmetric:
        return [f"{d1}/{ar}.{ai}.{br}.{bi}.las"]
    p1 = f"{d1}/{ar}.{ai}.{br}.{bi}.las"
    p2 = f"{d2}/{br}.{bi}.{ar}.{ai}.las"
    return [p2, p1] if bi < ai else [p1, p2]


def las_names2(aname, bname, base, symmetric):
    """daligner2's paths (pathLas / Write_Overlap_Buffer, dalign2/ovlbuffer.c:226-421): under
    <base>_<block>/, in (first, second) order."""
    def split(n):
        root, _, b = n.rpartition(".")
        return root, int(b)
    ar, ai = split(aname)
    br, bi = split(bname)
    p1 = "%s_%05d/%s.%d.%s.%d.las" % (base, ai, ar, ai, br, bi)
    if aname == bname or not symmetric:
        return [p1]
    p2 = "%s_%05d/%s.%d.%s.%d.las" % (base, bi, br, bi, ar, ai)
    return [p2, p1] if bi < ai else [p1, p2]


def write_las(path, recs, traces, tspace):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tb = 1 if tspace <= 125 else 2
    with open(path, "wb") as f:
        f.write(np.int64(len(recs)).tobytes())
        f.write(np.int32(tspace).tobytes())
        for r, t in zip(recs, traces):
            f.write(np.array([r["tlen"], r["diffs"], r["abpos"], r["bbpos"], r["aepos"], r["bepos"]], "<i4").tobytes())
            f.write(np.uint32(r["flags"]).tobytes())
            f.write(np.array([r["aread"], r["bread"], 0], "<i4").tobytes())
            f.write(np.asarray(t).astype("<u1" if tb == 1 else "<u2").tobytes())


def run(dbdir, flags, blocks, outdir, impl, wave_limit=None, variant=1, ctx_hook=None, stats_out=None):
    """Runs `daligner flags blocks[0] blocks[1]` (variant 2: `daligner2 -Pout ...`) with impl in
    {"oracle", "gpu"}; returns the paths.  wave_limit (gpu only) sets the widest band of the
    main aligner kernel (test hook); ctx_hook (gpu only) is called with the new context;
    stats_out (gpu only), a dict, receives the context's statistics after the run."""
    o = parse_flags(flags)
    aname, bname = blocks
    A = dazzdb.open_block(os.path.join(dbdir, aname))
    self_cmp = aname == bname
    B = A if self_cmp else dazzdb.open_block(os.path.join(dbdir, bname))
    for t in o["m"]:
        dazzdb.load_track(A, t)
        if not self_cmp:
            dazzdb.load_track(B, t)
    symmetric = not o["A"]
    mem = 0 if o["M"] is None else o["M"] * 0x40000000
    if self_cmp:
        last_read = A.ufirst + A.nreads - 1
    else:
        last_read = (B.ufirst + B.nreads - 1) if B.part < A.part else (A.ufirst + A.nreads - 1)
    tspace = o["s"]
    if impl == "oracle":
        import oracle
        p = oracle.make_params(A.freq, k=o["k"], w=o["w"], h=o["h"], t=o["t"], e=o["e"], l=o["l"], s=o["s"],
                               M=0, symmetric=symmetric, identity=o["I"], only_identity=o["O"], no_trace=o["T"],
                               H=o["H"], variant=variant, biased=o["b"])
        p.mem_limit = mem
        recs, traces, st = oracle.daligner(A, B, dazzdb.complement_block(B), p, self_cmp)
        if st["status"]:
            raise RuntimeError(f"oracle: daligner2 status {st['status']}")
    else:
        import marvel_b200 as mb
        ctx = mb.Context()
        if wave_limit is not None:
            ctx.set_wave_limit(wave_limit)
        if ctx_hook is not None:
            ctx_hook(ctx)
        if variant == 2:
            ctx.set_variant(2, o["H"])
        if o["b"]:
            ctx.set_biased(True)
        ctx.set_filter_params(o["k"], o["w"], o["t"], o["h"])
        ctx.new_align_spec(o["e"], o["s"], A.freq, symmetric, o["O"], o["T"])
        ctx.set_globals(2 * o["l"], o["I"] or o["O"], mem)
        ctx.load_block(0, A)
        if not self_cmp:
            ctx.load_block(1, B)
        if variant == 2:
            mb.run_loaded2(ctx, self_cmp)
        else:
            mb.run_loaded(ctx, self_cmp)
        r, tr = ctx.overlaps()
        if stats_out is not None:
            stats_out.update(ctx.stats())
        ctx.close()
        tb = 1 if tspace <= 125 else 2
        recs = r
        traces = [tr[int(x["toff"]):int(x["toff"]) + int(x["tlen"]) * tb].view("<u1" if tb == 1 else "<u2")
                  for x in r]
    names = las_names2(aname, bname, "out", symmetric) if variant == 2 else las_names(aname, bname, o["r"], symmetric)
    paths = [os.path.join(outdir, n) for n in names]
    if len(paths) == 1:
        write_las(paths[0], recs, traces, tspace)
    else:
        j = 0
        while j < len(recs) and recs[j]["aread"] <= last_read:
            j += 1
        write_las(paths[0], recs[:j], traces[:j], tspace)
        write_las(paths[1], recs[j:], traces[j:], tspace)
    return names

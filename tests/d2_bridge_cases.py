"""One-pair cases for daligner2's Handle_Redundancies (fusion + bridging): the harness's wire
format (oracle/d2_bridge_harness.c), the fixture file, and the oracle's entry point."""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np


@dataclasses.dataclass
class Case:
    a: np.ndarray          # A read, bases 0..3
    b: np.ndarray          # B read as the pair's alignment sees it (complemented when comp)
    tspace: int
    comp: int
    amatch: list           # [(hdr[6] = abpos bbpos aepos bepos diffs tlen, trace uint16), ...]
    bmatch: list | None    # the B-side paths, same length, or None


def _paths_bytes(ps):
    out = b""
    for h, t in ps:
        out += np.array(h, "<i4").tobytes() + np.asarray(t, "<u2").tobytes()
    return out


def encode(c: Case) -> bytes:
    hdr = np.array([c.a.size, c.b.size, c.tspace, c.comp, len(c.amatch), int(c.bmatch is not None)], "<i4")
    out = hdr.tobytes() + c.a.astype(np.uint8).tobytes() + c.b.astype(np.uint8).tobytes() + _paths_bytes(c.amatch)
    if c.bmatch is not None:
        out += _paths_bytes(c.bmatch)
    return out


def _read_paths(buf, off, n):
    ps = []
    for _ in range(n):
        h = [int(x) for x in np.frombuffer(buf, "<i4", 6, off)]
        off += 24
        t = np.frombuffer(buf, "<u2", h[5], off).copy()
        off += 2 * h[5]
        ps.append((h, t))
    return ps, off


def decode_results(buf: bytes, cases):
    """The harness output: per case (A-side paths kept, B-side paths kept or None)."""
    off, res = 0, []
    for c in cases:
        n = int(np.frombuffer(buf, "<i4", 1, off)[0])
        off += 4
        am, off = _read_paths(buf, off, n)
        bm = None
        if c.bmatch is not None:
            bm, off = _read_paths(buf, off, n)
        res.append((am, bm))
    assert off == len(buf)
    return res


def save(path, cases, expected):
    d = {}
    for i, (c, (am, bm)) in enumerate(zip(cases, expected)):
        d[f"a{i}"] = c.a
        d[f"b{i}"] = c.b
        d[f"m{i}"] = np.array([c.tspace, c.comp, int(c.bmatch is not None)], np.int32)
        for tag, ps in (("ia", c.amatch), ("ib", c.bmatch), ("oa", am), ("ob", bm)):
            if ps is None:
                continue
            d[f"{tag}h{i}"] = np.array([h for h, _ in ps], np.int32).reshape(-1, 6)
            d[f"{tag}t{i}"] = np.concatenate([t for _, t in ps]).astype(np.uint16) if ps else np.zeros(0, np.uint16)
    d["n"] = np.array([len(cases)])
    np.savez_compressed(path, **d)


def _paths(z, key, i):
    h = z[f"{key}h{i}"]
    t = z[f"{key}t{i}"]
    ps, o = [], 0
    for row in h:
        ps.append(([int(x) for x in row], t[o:o + int(row[5])]))
        o += int(row[5])
    return ps


def load(path):
    z = np.load(path)
    cases, expected = [], []
    for i in range(int(z["n"][0])):
        tspace, comp, has_b = (int(x) for x in z[f"m{i}"])
        c = Case(z[f"a{i}"], z[f"b{i}"], tspace, comp, _paths(z, "ia", i), _paths(z, "ib", i) if has_b else None)
        cases.append(c)
        expected.append((_paths(z, "oa", i), _paths(z, "ob", i) if has_b else None))
    return cases, expected


def was_bridged(c: Case, e) -> bool:
    """A kept path that is none of the inputs and is not one input extended over another
    by a plain fusion can only come from a bridge; counted for the fixture's statistics."""
    ins = {tuple(h) for h, _ in c.amatch}
    return any(tuple(h) not in ins for h, _ in e[0]) and len(e[0]) < len(c.amatch)


def flat(ps):
    hdr = np.array([h for h, _ in ps], np.int32).reshape(-1, 6)
    tr = np.concatenate([np.asarray(t, np.uint16) for _, t in ps]) if ps else np.zeros(0, np.uint16)
    return hdr, tr


def oracle_run(c: Case):
    """The oracle's Handle_Redundancies on a case: (A-side paths kept, B-side paths or None)."""
    import oracle
    L = oracle.lib()
    fn = L.or_handle_redundancies_d2
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    a = np.concatenate([[4], c.a, [4]]).astype(np.uint8)
    b = np.concatenate([[4], c.b, [4]]).astype(np.uint8)
    ps = c.amatch + (c.bmatch or [])
    hdr, tr = flat(ps)
    tcap = int(tr.size) + 4 * (max(c.a.size, c.b.size) // c.tspace + 8) * len(ps) + 1024
    oh = np.zeros((len(ps), 6), np.int32)
    ot = np.zeros(tcap, np.uint16)
    n = fn(a.ctypes.data + 1, b.ctypes.data + 1, c.a.size, c.b.size, c.tspace, c.comp, len(c.amatch),
           int(c.bmatch is not None), hdr.ctypes.data, tr.ctypes.data, oh.ctypes.data, ot.ctypes.data, tcap)
    assert n >= 0
    out, o = [], 0
    for i in range(n * (2 if c.bmatch is not None else 1)):
        h = [int(x) for x in oh[i]]
        out.append((h, ot[o:o + h[5]].copy()))
        o += h[5]
    return out[:n], (out[n:] if c.bmatch is not None else None)

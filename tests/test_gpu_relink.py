"""The link-time drop-in: the reference's own driver, dalign/daligner.c, compiled unmodified
and linked against libgpudalign.so in place of the reference's filter.c and align.c
(oracle/_ref/daligner_relinked, built by oracle/Makefile; the reference-named entry points
are marvel_b200/csrc/host/compat.c).  It must write every golden case's .las files as the
reference daligner does, and under -v print the reference's report character for
character."""
import glob
import os
import shutil
import subprocess

import pytest

from golden_cases import cases, load
from marvel_b200 import dazzdb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RELINKED = os.path.join(ROOT, "oracle", "_ref", "daligner_relinked")


def _copy_db(src, dst):
    for f in glob.glob(os.path.join(src, "*")) + glob.glob(os.path.join(src, ".*")):
        if os.path.isfile(f):
            shutil.copy(f, dst)


@pytest.fixture(scope="module")
def relinked():
    if not os.path.exists(RELINKED):
        pytest.skip("oracle/_ref/daligner_relinked was not built (make -C oracle ref needs the reference sources)")
    return RELINKED


@pytest.mark.parametrize("name", cases())
def test_reference_driver_relinked_writes_the_golden_las(relinked, name, tmp_path):
    d, meta = load(name)
    _copy_db(d, str(tmp_path))
    r = subprocess.run([relinked, "-j4"] + meta["flags"] + meta["blocks"], cwd=str(tmp_path), capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    for n in meta["las"]:
        ok, msg = dazzdb.las_equal(str(tmp_path / n), os.path.join(d, n))
        assert ok, f"{name} {n}: {msg}"


@pytest.mark.parametrize("name", ["self_s200_t20", "pair_blocks", "self_asym_lowmem", "pair_dust_biased"])
def test_reference_driver_relinked_verbose_report(relinked, name, tmp_path):
    d, meta = load(name)
    _copy_db(d, str(tmp_path))
    r = subprocess.run([relinked, "-v", "-j4"] + meta["flags"] + meta["blocks"], cwd=str(tmp_path),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    with open(os.path.join(d, "verbose.txt")) as f:
        assert r.stdout == f.read()


# ---- the single-alignment entry points, called by their reference names and signatures

def _abi():
    import ctypes as C

    import marvel_b200 as mb

    class Path(C.Structure):
        _fields_ = [("trace", C.c_void_p), ("tlen", C.c_int), ("diffs", C.c_int), ("abpos", C.c_int),
                    ("bbpos", C.c_int), ("aepos", C.c_int), ("bepos", C.c_int)]

    class Alignment(C.Structure):
        _fields_ = [("path", C.POINTER(Path)), ("flags", C.c_uint32), ("aseq", C.c_void_p), ("bseq", C.c_void_p),
                    ("alen", C.c_int), ("blen", C.c_int)]

    L = mb.lib()
    L.New_Align_Spec.restype = C.c_void_p
    L.New_Align_Spec.argtypes = [C.c_double, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int]
    L.New_Work_Data.restype = C.c_void_p
    L.Free_Work_Data.argtypes = [C.c_void_p]
    L.Local_Alignment.restype = C.POINTER(Path)
    L.Local_Alignment.argtypes = [C.POINTER(Alignment), C.c_void_p, C.c_void_p] + [C.c_int] * 5
    L.Compute_Trace_PTS.argtypes = [C.POINTER(Alignment), C.c_void_p, C.c_int, C.c_int, C.c_int]
    return C, L, Path, Alignment


def _bounded(seq):
    """A read with a 4 before and after it, as a loaded block holds it."""
    import numpy as np
    b = np.full(seq.size + 2, 4, np.uint8)
    b[1:-1] = seq
    return b


@pytest.mark.parametrize("comp", [0, 1])
def test_local_alignment_by_reference_name_matches_oracle(comp):
    import numpy as np
    import oracle
    C, L, Path, Alignment = _abi()
    d, _ = load("self_default")
    A = dazzdb.open_block(os.path.join(d, "G.1"))
    B = dazzdb.complement_block(A) if comp else A
    p = oracle.make_params(A.freq)
    h, _ = oracle.match_hits(A, A, p, True)
    rows = h[np.random.default_rng(5 + comp).choice(len(h), size=60, replace=False)]
    freq = (C.c_float * 4)(*[float(x) for x in A.freq])
    spec = L.New_Align_Spec(0.70, 100, freq, 4, 1, 0, 0)
    work = L.New_Work_Data()
    for diag, apos, ar, br in rows:
        a = _bounded(A.read(int(ar)))
        b = _bounded(B.read(int(br)))
        path = Path()
        al = Alignment(C.pointer(path), comp, a.ctypes.data + 1, b.ctypes.data + 1, a.size - 2, b.size - 2)
        anti = int(2 * apos - diag)
        bp = L.Local_Alignment(C.byref(al), work, spec, int(diag), int(diag), anti, -1, -1)
        assert bp, "Local_Alignment returned NULL"
        o, at, bt, _ = oracle.local_alignment(a, b, comp, int(diag), anti, p)
        got = [path.abpos, path.bbpos, path.aepos, path.bepos, path.diffs, path.tlen]
        bpath = bp.contents
        got += [bpath.abpos, bpath.bbpos, bpath.aepos, bpath.bepos, bpath.diffs, bpath.tlen]
        assert got == [int(x) for x in o]
        ta = np.ctypeslib.as_array(C.cast(path.trace, C.POINTER(C.c_uint16)), shape=(max(path.tlen, 1),))
        tb = np.ctypeslib.as_array(C.cast(bpath.trace, C.POINTER(C.c_uint16)), shape=(max(bpath.tlen, 1),))
        assert (ta[:path.tlen] == at).all() and (tb[:bpath.tlen] == bt).all()
    L.Free_Work_Data(work)


@pytest.mark.parametrize("name", ["self_default", "pair_blocks", "self_s200_t20"])
def test_compute_trace_pts_by_reference_name_matches_reference(name):
    """LAcheck -a's call (utils/LAcheck.c:232-249): reads loaded, B complemented for a COMP
    record, the record's trace points as uint16; the diffs must equal what the reference's
    own Compute_Trace_PTS computes (tests/golden/trace_pts.npz)."""
    import numpy as np
    C, L, Path, Alignment = _abi()
    fx = np.load(os.path.join(ROOT, "tests", "golden", "trace_pts.npz"))
    d, meta = load(name)
    G = dazzdb.open_block(os.path.join(d, "G"))
    Gc = dazzdb.complement_block(G)
    work = L.New_Work_Data()
    for las in meta["las"]:
        ts, recs, traces = dazzdb.read_las(os.path.join(d, las))
        want = fx[f"{name}/{las}"]
        for i in range(0, recs.size, 7):   # every 7th record: one device call each
            r = recs[i]
            a = _bounded(G.read(int(r["aread"])))
            b = _bounded((Gc if r["flags"] & 1 else G).read(int(r["bread"])))
            tr = np.ascontiguousarray(traces[i], np.uint16)
            path = Path(tr.ctypes.data, int(r["tlen"]), int(r["diffs"]), int(r["abpos"]), int(r["bbpos"]),
                        int(r["aepos"]), int(r["bepos"]))
            al = Alignment(C.pointer(path), int(r["flags"]), a.ctypes.data + 1, b.ctypes.data + 1, a.size - 2,
                           b.size - 2)
            assert L.Compute_Trace_PTS(C.byref(al), work, ts, 0, 0) == 0
            assert path.diffs == int(want[i]), (las, i, path.diffs, int(want[i]))
    L.Free_Work_Data(work)

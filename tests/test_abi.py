"""The C-ABI library loads and exports every entry point include/gpudalign.h declares (CPU)."""
import os
import re
import subprocess

import marvel_b200 as mb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "gpudalign.h")).read()
    return sorted(set(re.findall(r"\b(gd_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert sorted(mb.SYMBOLS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    L = mb.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s
    out = subprocess.run(["nm", "-D", "--defined-only", mb.LIBPATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    assert set(declared_symbols()) <= exported


def test_build_targets_sm100a_only():
    from marvel_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_no_gpu_fails_loudly_not_silently():
    import torch
    if torch.cuda.is_available():
        return
    try:
        mb.Context()
    except mb.GpuError as e:
        assert "no CUDA device" in str(e)
    else:
        raise AssertionError("Context() must refuse to run without a GPU")


def compat_symbols():
    txt = open(os.path.join(ROOT, "include", "gpudalign_compat.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Z][A-Za-z_]+)\s*\((?!\*)", txt)) - {"Path"})


def test_library_exports_the_reference_named_entry_points():
    """The reference-named interface (dalign/filter.h:67-73, dalign/align.h:131-344) a
    relinked reference driver resolves against libgpudalign.so."""
    names = compat_symbols()
    assert {"Set_Filter_Params", "Sort_Kmers", "Match_Filter", "New_Align_Spec", "Local_Alignment",
            "Compute_Trace_PTS", "Write_Overlap_Buffer", "Reset_Overlap_Buffer"} <= set(names)
    out = subprocess.run(["nm", "-D", "--defined-only", mb.LIBPATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    assert set(names) <= exported, set(names) - exported
    # the driver globals are weak references: the library loads without them
    weak = subprocess.run(["nm", "-D", mb.LIBPATH], capture_output=True, text=True).stdout
    for g in ("VERBOSE", "BIASED", "MINOVER", "IDENTITY", "MEM_LIMIT", "MEM_PHYSICAL"):
        assert any(line.split()[-2:] == ["w", g] for line in weak.splitlines()), g

"""Builds libgpudalign.so (the sm_100a overlap path + its C ABI) in-tree with nvcc."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgpudalign.so")
CLI = os.path.join(HERE, "daligner_gpu")
CLI2 = os.path.join(HERE, "daligner2_gpu")
SOURCES = ["gd_prims.cu", "gd_filter.cu", "gd_filter2.cu", "gd_align.cu", "gd_pipeline.cu", "gd_noalloc.cu", "gd_verify.cu", "gd_triage.cu", "gd_output.cu", "gd_dust.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h", ".c"))]
    deps.append(os.path.join(ROOT, "include", "gpudalign.h"))
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    if force or _stale(LIB, deps):
        objs = []
        for s in SOURCES:
            o = os.path.join(objdir, s.replace(".cu", ".o"))
            cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, s), "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(o)
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    for cli, main in ((CLI, "daligner_main.c"), (CLI2, "daligner2_main.c")):
        cli_src = os.path.join(CSRC, "host", main)
        if force or _stale(cli, [cli_src, LIB, os.path.join(CSRC, "host", "dazz_db.c")]):
            cmd = ["gcc", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), "-o", cli, cli_src,
                   os.path.join(CSRC, "host", "dazz_db.c"), "-L" + HERE, "-lgpudalign", "-lm", "-Wl,-rpath,$ORIGIN"]
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)

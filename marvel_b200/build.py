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
# host C in the library: the reference-named entry points and the -v report they share with the command line
HOST_SOURCES = ["host/compat.c", "host/gd_report.c"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    deps = [os.path.join(d, f) for d, _, fs in os.walk(CSRC) for f in fs if f.endswith((".cu", ".cuh", ".h", ".c"))]
    deps.append(os.path.join(ROOT, "include", "gpudalign.h"))
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    if force or _stale(LIB, deps):
        cmds, objs = [], []
        for s in SOURCES:
            o = os.path.join(objdir, s.replace(".cu", ".o"))
            cmds.append([NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, s), "-o", o])
            objs.append(o)
        for s in HOST_SOURCES:
            o = os.path.join(objdir, os.path.basename(s).replace(".c", ".o"))
            cmds.append(["gcc", "-O2", "-Wall", "-fPIC", "-std=gnu11", "-I" + os.path.join(ROOT, "include"),
                         "-I" + os.path.join(CSRC, "host"), "-c", os.path.join(CSRC, s), "-o", o])
            objs.append(o)
        # the translation units compile independently: in parallel, the largest first
        from concurrent.futures import ThreadPoolExecutor
        cmds.sort(key=lambda c: -os.path.getsize(c[c.index("-c") + 1]))
        with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
            for cmd, rc in zip(cmds, ex.map(lambda c: subprocess.run(c).returncode, cmds)):
                if verbose:
                    print(" ".join(cmd))
                if rc:
                    raise subprocess.CalledProcessError(rc, cmd)
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    for cli, main in ((CLI, "daligner_main.c"), (CLI2, "daligner2_main.c")):
        cli_src = os.path.join(CSRC, "host", main)
        if force or _stale(cli, [cli_src, LIB, os.path.join(CSRC, "host", "dazz_db.c")]):
            cmd = ["gcc", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CSRC, "host"),
                   "-o", cli, cli_src,
                   os.path.join(CSRC, "host", "dazz_db.c"), "-L" + HERE, "-lgpudalign", "-lm", "-Wl,-rpath,$ORIGIN"]
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)

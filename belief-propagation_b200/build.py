"""Build lib/libbp.so: the drop-in graph API + CUDA engine, sm_100a only.

    python belief-propagation_b200/build.py [--verbose-ptxas] [--force]

nvcc compiles the .cu sources for sm_100a (-gencode arch=compute_100a,
code=sm_100a); gcc compiles the C host sources without FMA contraction (the
host-side send_message keeps the reference's rounding); nvcc links one shared
library with the CUDA runtime linked statically, so the library needs no
CUDA runtime on the library path at load time.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libbp.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["engine.cu", "loopy.cu", "tree.cu", "levels_gpu.cu", "batch.cu", "unrolled.cu"]
C_SOURCES = ["graph_api.c", "levels.c", "xmlbif.c"]
HEADERS = ["bp_internal.h", "bp_device.cuh", "bp_levels.h", "bp_serial.cuh", "flood_split.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(force=False, verbose_ptxas=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    common_deps = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INCLUDE, h) for h in ("bp.h", "graph.h", "constants.h", "xml-expression.h")]
    steps = []
    objs = []
    for s in CU_SOURCES:
        o = os.path.join(OBJ, s.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [os.path.join(CSRC, s)] + common_deps):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC, "-c",
                   "-o", o, os.path.join(CSRC, s)]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            steps.append(cmd)
    for s in C_SOURCES:
        o = os.path.join(OBJ, s.replace(".c", ".o"))
        objs.append(o)
        if force or _newer(o, [os.path.join(CSRC, s)] + common_deps):
            steps.append(["gcc", "-O3", "-fPIC", "-std=gnu99", "-ffp-contract=off", "-Wall",
                          "-I", INCLUDE, "-I", CSRC, "-c", "-o", o, os.path.join(CSRC, s)])
    out = ""
    if steps:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for text in ex.map(_run, steps):
                out += text
    if force or steps or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-Xlinker", "-Bsymbolic",
              "-o", LIB, *objs, "-lrt", "-lpthread", "-ldl"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    out = build(force=a.force, verbose_ptxas=a.verbose_ptxas)
    if a.verbose_ptxas:
        print(out)
    print(LIB)


if __name__ == "__main__":
    main()

"""Build recipe of the CUDA library: nvcc for sm_100a, in-tree.

    python -m sfemans_b200.build          # -> sfemans_b200/_lib/libsfemans_nl.so

The shared library is the product: a C-ABI (include/sfemans_nl.h) over the
CUDA kernels in sfemans_b200/csrc.  It links only the CUDA runtime.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libsfemans_nl.so")
SOURCES = ["sfnl_capi.cu", "sfnl_grid.cu", "sfnl_fast.cu", "sfnl_large.cu", "sfnl_split.cu", "sfnl_synth.cu",
           "sfnl_gauss.cu", "sfnl_probe.cu", "sfnl_r3.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    objs, cmds = [], []
    for s in SOURCES:
        src = os.path.join(SRC, s)
        obj = os.path.join(OUT_DIR, s.replace(".cu", ".o"))
        deps = [src] + [os.path.join(SRC, h) for h in os.listdir(SRC) if h.endswith((".cuh", ".h"))]
        deps.append(os.path.join(os.path.dirname(HERE), "include", "sfemans_nl.h"))
        if not os.path.exists(obj) or any(os.path.getmtime(d) > os.path.getmtime(obj) for d in deps):
            cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                   "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd))
            cmds.append(cmd)
        objs.append(obj)
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs]  # static cudart (nvcc default)
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))

"""Build the B200 simulation core into neuro_edit_v2_b200/_lib/libne2b.so.

Compiles the CUDA kernels ahead of time for sm_100a only
(`-gencode arch=compute_100a,code=sm_100a`) with `-fmad=false`, so no float
operation of the step is contracted into an FMA, and the host sources with
`-ffp-contract=off`.  The library is built in-tree so it travels with the
repository; nothing is installed.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libne2b.so")
SOURCES = ["ne2b_step_k00.cu", "ne2b_step_k01.cu", "ne2b_step_k10.cu", "ne2b_step_k11.cu", "ne2b_kernels.cu",
           "ne2b_engine.cu", "ne2b_capi.cu", "ne2b_noalloc.cu", "ne2b_csr.cu", "ne2b_readout.cu", "ne2b_host.cpp",
           "ne2b_ne2.cpp"]
HEADERS = ["ne2b_device.cuh", "ne2b_layout.h", "ne2b_kernels.h", "ne2b_engine.h", "ne2b_handles.h", "ne2b_parallel.h",
           "ne2b_step.cuh", "ne2b_step_kind.h", "ne2b_net.h", "ne2b_csr.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fno-fast-math",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "ne2b.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run_all(cmds, verbose: bool) -> None:
    """Run the compiler commands concurrently; raise on the first failure."""
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmds = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        cmds.append([nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    _run_all(cmds, verbose)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp, "-lcudart",
           "-Xcompiler", "-pthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

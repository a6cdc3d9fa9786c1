"""Builds the CUDA library ``librtspatial_b200.so`` in-tree for sm_100a.

The library is the product: the C-ABI declared in ``include/rtspatial_b200.h``
and implemented by ``csrc/*.cu``.  Fast-math is never enabled: the
range-intersects predicate relies on IEEE division and separately rounded
products.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librtspatial_b200.so")
SOURCES = ["rts_query_occ1.cu", "rts_query_occ2.cu", "rts_query_occ3.cu", "rts_query_occ4.cu",
           "rts_query_staged.cu",
           "rts_index.cu", "rts_plan.cu", "rts_server.cu", "rts_tune.cu", "rts_frontier.cu",
           "rts_query.cu", "rts_build.cu", "rts_memory.cu"]
HEADERS = ["rts_device.cuh", "rts_traverse.cuh", "rts_query_kernels.cuh", "rts_internal.h",
           "rts_index_impl.h", "rts_handler_kernel.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
    "-fmad=false",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "rtspatial_b200.h"))
    deps.append(__file__)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the shared library if any source is newer; returns its path."""
    if not force and not _stale():
        return LIB
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, "_" + src.replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(obj)
    # one nvcc per source, in parallel (the query kernels, one source per
    # occupancy, dominate)
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                           *objs, "-o", tmp])
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

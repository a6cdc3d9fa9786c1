"""Compiles a handler module: this library's query kernels with the caller's
own per-pair device handlers (``rtspatial_handle_*``), for builds without
CMake.  The same command as ``RTSPATIAL_COMPILE_SHADERS`` in
``cmake/rtspatial_shaders.cmake``.

    python -m rtspatial_b200.handlers <handler header> <output dir> [-I <dir>]...

writes ``<output dir>/rtspatial_handlers.cubin``; load it with
``rts_load_handler_module`` (or ``SpatialIndex.load_handler_module``, or
``rtspatial::Config::ptx_root = <output dir>`` in C++).
"""
from __future__ import annotations

import argparse
import os
import subprocess

from .build import nvcc

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCE = os.path.join(HERE, "shaders", "rts_handler_module.cu")
MODULE_FILE = "rtspatial_handlers.cubin"


def compile_module(header: str, out_dir: str, include_dirs=(), force: bool = False) -> str:
    """Compiles the handler module for `header` into out_dir; returns the
    cubin's path.  Skips the compile when the cubin is newer than its inputs
    (unless `force`)."""
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, MODULE_FILE)
    compat = os.path.join(out_dir, "compat")
    os.makedirs(compat, exist_ok=True)
    stub = os.path.join(compat, "optix.h")
    if not os.path.exists(stub):
        with open(stub, "w") as f:
            f.write("/* Empty: handler headers written for RTSpatial include <optix.h> but use "
                    "nothing from it. */\n")
    hdr = os.path.abspath(header)
    deps = [SOURCE, hdr] + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))
                            if f.endswith((".cuh", ".h"))]
    if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out)
                                                  for d in deps if os.path.exists(d)):
        return out
    cmd = [nvcc(), "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3",
           "-fmad=false", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc"),
           "-I", os.path.dirname(hdr)]
    for d in include_dirs:
        cmd += ["-I", d]
    cmd += ["-I", compat, "-include", hdr, SOURCE, "-o", out + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("header")
    ap.add_argument("out_dir")
    ap.add_argument("-I", dest="include", action="append", default=[])
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(compile_module(a.header, a.out_dir, a.include, a.force))


if __name__ == "__main__":
    main()

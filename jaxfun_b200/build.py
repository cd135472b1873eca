"""In-tree build of libjfb200.so for sm_100a (nvcc, explicit -gencode).

The library is built next to this file so that it travels with the source
tree; nothing is installed into site-packages or a JIT cache.
"""

from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libjfb200.so")
SOURCES = ["jfb_la.cu", "jfb_kmm.cu", "jfb_kmm_setup.cpp"]
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


STAMPS_OUT = os.path.join(HERE, "libjfb200_stamps.so")


def build(force: bool = False, verbose: bool = False, stamps: bool = False) -> str:
    """Compile the CUDA sources into ``libjfb200.so`` if any source is newer.

    ``stamps=True`` builds ``libjfb200_stamps.so`` instead: the same library
    with -DJFB_PHASE_STAMPS, whose step kernels record global-timer stamps
    at their phase boundaries (``jfb_debug_read_stamps``; load it with
    JFB200_LIB pointing at it).  For profiling only."""
    out = STAMPS_OUT if stamps else OUT
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [
        os.path.join(CSRC, f)
        for f in os.listdir(CSRC)
        if f.endswith((".cuh", ".h"))
    ] + [os.path.join(HERE, "..", "include", "jfb200.h")]
    if not force and os.path.exists(out):
        out_mtime = os.path.getmtime(out)
        if all(os.path.getmtime(d) <= out_mtime for d in deps):
            return out
    cmd = [nvcc(), *FLAGS, *(["-DJFB_PHASE_STAMPS"] if stamps else []), "-o", out, *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    import sys

    build(force=True, verbose=True, stamps="--stamps" in sys.argv)

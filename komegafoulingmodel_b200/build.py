"""Build recipe of the native library (libkofm.so, sm_100a).

    python -m komegafoulingmodel_b200.build

compiles csrc/kofm_api.cu (which includes the kernel headers) with nvcc for
sm_100a into komegafoulingmodel_b200/libkofm.so, next to this file, so the
library travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libkofm.so")
SOURCES = ["kofm_api.cu", "kofm_noalloc.cu"]
DEPS = ["kofm_api.cu", "kofm_noalloc.cu", "kofm_common.cuh", "kofm_lb.cuh",
        "kofm_komega.cuh", "kofm_gmres.cuh", "kofm_komega_api.inc"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    paths = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(ROOT, "include", "kofm.h")]
    return any(os.path.getmtime(p) > t for p in paths if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"),
           "-I", CSRC, "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)

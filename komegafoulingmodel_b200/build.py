"""Build recipe of the native library (libkofm.so, sm_100a).

    python -m komegafoulingmodel_b200.build

compiles csrc/kofm_api.cu (which includes the kernel headers) with nvcc for
sm_100a into komegafoulingmodel_b200/libkofm.so, next to this file, so the
library travels with the source tree; then the host classes (host/) into
libkofm_host.so and the step-loop driver host/kofm_host_run, both linked
against libkofm.so.
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
        "kofm_komega.cuh", "kofm_gmres.cuh", "kofm_sstep.cuh", "kofm_komega_api.inc",
        "kofm_batch.inc", "kofm_thermal.cuh", "kofm_thermal_api.inc", "kofm_adjoint.inc",
        "kofm_geometry.inc"]


def _all_sources() -> list[str]:
    """Every file of csrc/ (a new header can never be missed)."""
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))]

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
    paths = _all_sources() + [os.path.join(ROOT, "include", "kofm.h")]
    return any(os.path.getmtime(p) > t for p in paths if os.path.exists(p))


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libkofm_host.so")
HOST_RUN = os.path.join(HOST, "kofm_host_run")
HOST_SOURCES = ["kofm_host.cpp", "kofm_host.hpp", "kofm_host_run.cpp"]


def host_needs_build() -> bool:
    outs = [HOST_LIB, HOST_RUN]
    if not all(os.path.exists(o) for o in outs):
        return True
    t = min(os.path.getmtime(o) for o in outs)
    paths = [os.path.join(HOST, s) for s in HOST_SOURCES] + [os.path.join(ROOT, "include", "kofm.h"), LIB]
    return any(os.path.getmtime(p) > t for p in paths if os.path.exists(p))


def build_host(force: bool = False, verbose: bool = False) -> str:
    """g++ build of the host classes and the driver (rpath $ORIGIN)."""
    if not force and not host_needs_build():
        return HOST_LIB
    cxx = os.environ.get("KOFM_CXX", "g++")
    inc = ["-I", os.path.join(ROOT, "include"), "-I", HOST]
    cmds = [
        (HOST_LIB, [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", *inc, "-o", HOST_LIB + ".tmp",
                    os.path.join(HOST, "kofm_host.cpp"), "-L", HERE, "-lkofm", "-Wl,-rpath,$ORIGIN"]),
        (HOST_RUN, [cxx, "-O2", "-std=c++17", *inc, "-o", HOST_RUN + ".tmp",
                    os.path.join(HOST, "kofm_host_run.cpp"), "-L", HERE, "-lkofm_host", "-lkofm",
                    "-Wl,-rpath,$ORIGIN/.."]),
    ]
    for out, cmd in cmds:
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)
    return HOST_LIB


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not needs_build():
        build_host(force=False, verbose=verbose)
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"),
           "-I", CSRC, "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    build_host(force=True, verbose=verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)

"""Build the sm_100a shared library of the B200 search path (in-tree).

    python -m dummest_b200.build            # -> dummest_b200/libdummest_b200.so

The library is compiled with nvcc for sm_100a only.  Float arithmetic uses
flush-to-zero (the reference engine sets FTZ/DAZ on every thread,
dummest-core.hh:143-154) and no automatic multiply-add contraction: every
fused multiply-add in the kernels is written out explicitly, in the
association order of the reference recurrences.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdummest_b200.so")

SOURCES = ["dmst_api.cu", "host_model.cpp", "windows.cpp"]
HEADERS = ["dp_common.cuh", "dp_wavefront.cuh", "dp_exact.cuh", "dp_exact_wave.cuh", "null_model.cuh", "host_model.h",
           "dp_adjoint.cuh", "dp_posterior.cuh", "dp_search.cuh", "dp_traceback.cuh", "dp_traceback_job.cuh",
           "dp_stagger.cuh", "dp_plain.cuh"]

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-ftz=true",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-O2",
    "-Xptxas", "-v" if os.environ.get("DMST_PTXAS_VERBOSE") else "-O3",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "dummest_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, out: str = LIB, defines: tuple = ()) -> str:
    if not force and out == LIB and not needs_build():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", out]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libdummest_b200.so")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

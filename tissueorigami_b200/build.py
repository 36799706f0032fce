"""Build the CUDA library ``tissueorigami_b200/_lib/libtf_b200.so`` for sm_100a with nvcc.

The library is built in-tree (no JIT cache) so the same file is loaded by tests, the benchmark
and a host application that links it.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libtf_b200.so")
SOURCES = ["csrc/tf_capi.cu", "csrc/tf_element.cu", "csrc/tf_krylov.cu", "csrc/tf_noalloc.cu",
           "csrc/tf_adjoint.cu", "csrc/tf_direct.cu", "csrc/tf_bench.cu", "csrc/tf_dense.cu",
           "csrc/tf_multilevel.cu", "csrc/tf_packing.cu", "csrc/tf_lumen.cu"]
LIBS = ["-lcusolver", "-lcusparse"]  # tf_direct.cu only: the sparse direct solve timed beside the Krylov solve
HEADERS = ["csrc/tf_internal.cuh", "../include/tf_b200.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build tissueorigami_b200")


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if it is missing or older than its sources; return its path."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", tmp, *SOURCES, *LIBS]
    res = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))

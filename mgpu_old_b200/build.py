"""Build libmgpusort_b200.so in-tree with nvcc for sm_100a.

The library is the product: the C ABI of include/mgpusort.h and
include/mgpusort_b200.h over the kernels in csrc/. It is built next to this
file so that it travels with the source tree; nothing is installed.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB_NAME = "libmgpusort_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

SOURCES = [
    "engine.cpp",
    "sort_kernels.cu",
    "onesweep.cu",
    "noalloc.cu",
    "server.cpp",
    "bwt.cu",
]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES]
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                files.append(os.path.join(d, f))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def _compile(lib_path: str, objdir: str, defines: dict | None, verbose: bool) -> str:
    os.makedirs(objdir, exist_ok=True)
    extra = [f"-D{k}={v}" for k, v in (defines or {}).items()]
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", INCLUDE, "-c", os.path.join(CSRC, src),
               "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = lib_path + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
           "-Xcompiler", "-fPIC", *objs, "-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib_path)
    return lib_path


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source into the shared library; return its path."""
    if not force and up_to_date():
        return LIB_PATH
    return _compile(LIB_PATH, os.path.join(HERE, "_build"), None, verbose)


def build_variant(name: str, defines: dict, verbose: bool = False) -> str:
    """The library with tile_config.h values overridden by `defines`, built
    under _build/tune/<name>/ (for the autotuner); returns its path."""
    d = os.path.join(HERE, "_build", "tune", name)
    return _compile(os.path.join(d, LIB_NAME), d, defines, verbose)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

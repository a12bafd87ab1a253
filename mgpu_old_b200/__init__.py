"""B200-native stable radix sort with Modern GPU's sortArray C API.

The product is libmgpusort_b200.so (C ABI: include/mgpusort.h and
include/mgpusort_b200.h), built in-tree by mgpu_old_b200.build from the CUDA
and C++ sources in csrc/. This package adds a ctypes mirror of that API
(mgpu_old_b200.api) for Python callers, tests and benchmarks.
"""
from . import build  # noqa: F401

__all__ = ["build", "api"]

"""ctypes binding of liboracle.so (oracle.cpp) and of the reference's own CPU
code built into _ref/: its radix sort demo (ref_cpusort_shim.cpp) and its BWT
library's string quicksort (ref_bwt_shim.cpp). TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_int, c_size_t, c_uint, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_cpusort.so")
REF_BWT_LIB = os.path.join(HERE, "_ref", "libref_bwt.so")
# Where the reference project's sources lie (read-only; only its CPU files
# are compiled, by the Makefile's `ref` target). MGPU_REFERENCE_TREE
# overrides the default location; where the tree is absent, the _ref/
# libraries are not built and the tests pinned to them are skipped.
REFERENCE_TREE = os.environ.get("MGPU_REFERENCE_TREE", "/root/reference")

_u32p = POINTER(c_uint)


def build(ref: bool = True) -> None:
    """make liboracle.so, and _ref/ when the reference tree is present."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref and os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_TREE}"],
                       check=True)


_lib = None
_ref = None
_ref_bwt = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build(ref=False)
        l = ctypes.CDLL(LIB)
        l.oracle_sort_stable.restype = c_int
        l.oracle_sort_stable.argtypes = [_u32p, POINTER(_u32p), c_int, c_int, c_int,
                                         c_int, _u32p, POINTER(_u32p)]
        l.oracle_sort_lsd.restype = c_int
        l.oracle_sort_lsd.argtypes = [_u32p, POINTER(_u32p), c_int, c_int, c_int,
                                      POINTER(c_int), c_int, c_int, c_int]
        l.oracle_sort_segments.restype = c_int
        l.oracle_sort_segments.argtypes = [_u32p, POINTER(_u32p), c_int, POINTER(c_int),
                                           c_int, c_int, c_int, _u32p, POINTER(_u32p)]
        l.oracle_std_sort_keys.restype = None
        l.oracle_std_sort_keys.argtypes = [_u32p, c_int]
        l.oracle_reference_ex_plan.restype = c_int
        l.oracle_reference_ex_plan.argtypes = [c_int, c_int, POINTER(c_int)]
        l.oracle_bwt.restype = c_int
        l.oracle_bwt.argtypes = [c_void_p, c_int, c_int, POINTER(c_int), c_void_p,
                                 POINTER(c_int), POINTER(ctypes.c_float)]
        _lib = l
    return _lib


def ref_lib() -> ctypes.CDLL | None:
    """The reference's cpusort.cpp built here, or None where it is absent."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        r = ctypes.CDLL(REF_LIB)
        r.ref_cpusort_sort1.argtypes = [_u32p, c_size_t]
        r.ref_cpusort_sort2.argtypes = [_u32p, c_size_t, c_uint]
        r.ref_cpusort_sort2pass.argtypes = [_u32p, c_uint, c_uint, c_size_t, c_uint]
        _ref = r
    return _ref


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_u32p)


def _ptrs(arrays):
    arr = (_u32p * 6)()
    for i, a in enumerate(arrays):
        arr[i] = _p(a)
    return arr


def sort_stable(keys: np.ndarray, values: list[np.ndarray] | None, value_count: int,
                first_bit: int, end_bit: int):
    """Stable sort by the bit field; returns (keys, [values])."""
    n = keys.size
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    vals = [np.ascontiguousarray(v, dtype=np.uint32) for v in (values or [])]
    arrays = 1 if value_count == -1 else value_count
    kout = np.empty(n, np.uint32)
    vout = [np.empty(n, np.uint32) for _ in range(arrays)]
    rc = lib().oracle_sort_stable(_p(keys), _ptrs(vals), value_count, n, first_bit,
                                  end_bit, _p(kout), _ptrs(vout))
    if rc:
        raise ValueError("oracle_sort_stable: invalid arguments")
    return kout, vout


def sort_lsd(keys: np.ndarray, values: list[np.ndarray] | None, value_count: int,
             first_bit: int, widths: list[int], block_size: int = 2048,
             threads: int = 1):
    """Blocked LSD radix sort (cpusort.cpp:122-186 generalised); returns copies."""
    keys = np.array(keys, dtype=np.uint32, copy=True)
    arrays = 1 if value_count == -1 else value_count
    if value_count == -1:
        vals = [np.empty(keys.size, np.uint32)]
    else:
        vals = [np.array(v, dtype=np.uint32, copy=True) for v in (values or [])]
    w = (c_int * max(1, len(widths)))(*widths)
    rc = lib().oracle_sort_lsd(_p(keys), _ptrs(vals), value_count, keys.size,
                               first_bit, w, len(widths), block_size, threads)
    if rc:
        raise ValueError("oracle_sort_lsd: invalid arguments")
    return keys, vals[:arrays]


def sort_segments(keys: np.ndarray, values: list[np.ndarray] | None, value_count: int,
                  offsets: np.ndarray, first_bit: int, end_bit: int):
    """Each segment sorted on its own (one sortArray per segment)."""
    keys = np.ascontiguousarray(keys, dtype=np.uint32)
    vals = [np.ascontiguousarray(v, dtype=np.uint32) for v in (values or [])]
    offs = np.ascontiguousarray(offsets, dtype=np.int32)
    arrays = 1 if value_count == -1 else value_count
    kout = np.empty(keys.size, np.uint32)
    vout = [np.empty(keys.size, np.uint32) for _ in range(arrays)]
    rc = lib().oracle_sort_segments(_p(keys), _ptrs(vals), value_count,
                                    offs.ctypes.data_as(POINTER(c_int)), offs.size - 1,
                                    first_bit, end_bit, _p(kout), _ptrs(vout))
    if rc:
        raise ValueError("oracle_sort_segments: invalid arguments")
    return kout, vout


def reference_ex_plan(num_bits: int, bit_pass: int) -> list[int]:
    w = (c_int * 32)()
    n = lib().oracle_reference_ex_plan(num_bits, bit_pass, w)
    return list(w[:n])


def std_sort_keys(keys: np.ndarray) -> np.ndarray:
    out = np.array(keys, dtype=np.uint32, copy=True)
    lib().oracle_std_sort_keys(_p(out), out.size)
    return out


def bwt(block, key_size: int):
    """(indices, transform, segCount, avSegSize) of the block's rotations
    (oracle_bwt)."""
    data = np.frombuffer(bytes(block), dtype=np.uint8) if not hasattr(block, "dtype") \
        else np.ascontiguousarray(block, dtype=np.uint8)
    n = int(data.size)
    idx = np.zeros(max(n, 1), dtype=np.int32)
    xf = np.zeros(max(n, 1), dtype=np.uint8)
    seg = c_int(0)
    av = ctypes.c_float(0)
    rc = lib().oracle_bwt(data.ctypes.data_as(c_void_p), n, int(key_size),
                          idx.ctypes.data_as(POINTER(c_int)), xf.ctypes.data_as(c_void_p),
                          ctypes.byref(seg), ctypes.byref(av))
    if rc:
        raise ValueError("oracle_bwt: invalid arguments")
    return idx[:n], xf[:n], seg.value, av.value


def ref_bwt_lib() -> ctypes.CDLL | None:
    """The reference BWT library's cpusort.cpp built here, or None."""
    global _ref_bwt
    if _ref_bwt is None and os.path.exists(REF_BWT_LIB):
        r = ctypes.CDLL(REF_BWT_LIB)
        r.ref_bwt_qsort_strings.restype = None
        r.ref_bwt_qsort_strings.argtypes = [POINTER(c_int), POINTER(c_int), c_void_p, c_int]
        _ref_bwt = r
    return _ref_bwt


def ref_bwt_block(block):
    """Rotation order and transform of a block by the reference's own host
    block sort: QSortStrings over every rotation of the doubled block, as its
    TinyBlockSort does (bwt/src/mgpubwt/mgpubwt.cpp:180-205)."""
    r = ref_bwt_lib()
    if r is None:
        return None
    data = np.ascontiguousarray(np.frombuffer(bytes(block), dtype=np.uint8)
                                if not hasattr(block, "dtype") else block, dtype=np.uint8)
    n = int(data.size)
    sym = np.concatenate([data, data])
    idx = np.arange(n, dtype=np.int32)
    if n >= 2:
        base = idx.ctypes.data_as(POINTER(c_int))
        last = ctypes.cast(ctypes.addressof(base.contents) + 4 * (n - 1), POINTER(c_int))
        r.ref_bwt_qsort_strings(base, last, sym.ctypes.data_as(c_void_p), n)
    xf = sym[(idx.astype(np.int64) + n - 1)]
    return idx, xf

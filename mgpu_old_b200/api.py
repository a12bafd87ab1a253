"""Python mirror of the sort library's C API (ctypes over libmgpusort_b200.so).

The names follow Modern GPU's C API and C++ wrappers: the sortStatus_t codes
and sortStatusString (inc/mgpusort.h:21-39), the sortData_d struct
(inc/mgpusort.h:63-147), the engine functions (inc/mgpusort.h:50-187) and the
RAII helpers MgpuException / MgpuSortData / MgpuSort (inc/mgpusort.hpp:12-114).
Every call goes through the C ABI; there is no fallback. If the library has
not been built, importing this module raises.
"""
from __future__ import annotations

import ctypes
import enum
import os
from ctypes import POINTER, c_bool, c_char_p, c_int, c_uint, c_uint64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmgpusort_b200.so")


class SortStatus(enum.IntEnum):
    """sortStatus_t, same order and values as inc/mgpusort.h:21-36."""
    SUCCESS = 0
    NOT_INITIALIZED = 1
    DEVICE_ALLOC_FAILED = 2
    HOST_ALLOC_FAILED = 3
    CONFIG_NOT_SUPPORTED = 4
    CONTEXT_MISMATCH = 5
    INVALID_CONTEXT = 6
    KERNEL_NOT_FOUND = 7
    KERNEL_ERROR = 8
    LAUNCH_ERROR = 9
    INVALID_VALUE = 10
    DEVICE_ERROR = 11
    INTERNAL_ERROR = 12
    UNSUPPORTED_DEVICE = 13


class SortData(ctypes.Structure):
    """sortData_d (inc/mgpusort.h:63-147), CUdeviceptr view of the unions.

    values[i] is the pair of buffers of value array i+1 (values1..values6).
    """
    _fields_ = [
        ("maxElements", c_int),
        ("numElements", c_int),
        ("valueCount", c_int),
        ("firstBit", c_int),
        ("endBit", c_int),
        ("preserveEndKeys", c_bool),
        ("earlyExit", c_bool),
        ("parity", c_int),
        ("keys", c_uint64 * 2),
        ("values", (c_uint64 * 2) * 6),
    ]


class ServerConfig(ctypes.Structure):
    """sortServerConfig (mgpusort_b200.h)."""
    _fields_ = [
        ("memoryBudget", ctypes.c_size_t),
        ("slots", c_int),
        ("coalesceMax", c_int),
        ("maxBatchElements", c_int),
        ("maxBatchRequests", c_int),
    ]


assert ctypes.sizeof(SortData) == 144
assert SortData.keys.offset == 32 and SortData.values.offset == 48

EXPORTED_SYMBOLS = (
    # inc/mgpusort.h (sort/src/mgpusort/mgpusort.def:3-18)
    "sortStatusString", "sortCreateEngine", "sortLoadKernel", "sortIncEngine",
    "sortReleaseEngine", "sortCreateData", "sortDestroyData", "sortAllocData",
    "sortFreeData", "sortArray", "sortArrayEx", "sortHost", "sortDevice",
    # mgpusort_b200.h (no reference counterpart)
    "sortArrayAsync", "sortSynchronize", "sortPlanPasses", "sortInjectFault",
    "sortEnableKernelTiming", "sortReadKernelTiming", "sortArrayNoAlloc",
    "sortSegmentedArray", "sortArrayTyped", "sortSelectKey", "sortEnableGraphs",
    "sortGraphStats", "sortServerCreate", "sortServerSubmit", "sortServerPoll",
    "sortServerWait", "sortServerDestroy",
    # mgpubwt.h (inc/mgpubwt.h, bwt/src/mgpubwt/bwt.def)
    "bwtStatusString", "bwtCreateEngine", "bwtDestroyEngine", "bwtSortBlock",
)

# sortKeyType_t of sortArrayTyped.
KEY_UINT32, KEY_INT32, KEY_FLOAT32 = 0, 1, 2

# Largest numElements accepted by sortArrayNoAlloc (SORT_NOALLOC_MAX_ELEMENTS).
NOALLOC_MAX_ELEMENTS = 4194304

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the library and declare every signature. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is not built; run `python -m mgpu_old_b200.build` first")
    lib = ctypes.CDLL(path)
    engine_t = c_void_p
    data_t = POINTER(SortData)
    sigs = {
        "sortStatusString": (c_char_p, [c_int]),
        "sortCreateEngine": (c_int, [c_char_p, POINTER(engine_t)]),
        "sortLoadKernel": (c_int, [engine_t, c_int, c_int, c_bool, c_int]),
        "sortIncEngine": (c_int, [engine_t]),
        "sortReleaseEngine": (c_int, [engine_t]),
        "sortCreateData": (c_int, [engine_t, c_int, c_int, POINTER(data_t)]),
        "sortDestroyData": (c_int, [data_t]),
        "sortAllocData": (c_int, [engine_t, data_t]),
        "sortFreeData": (c_int, [data_t]),
        "sortArray": (c_int, [engine_t, data_t]),
        "sortArrayEx": (c_int, [engine_t, data_t, c_int, c_int, c_int, c_bool]),
        "sortHost": (c_int, [engine_t, POINTER(c_uint), POINTER(c_uint), c_int, c_int]),
        "sortDevice": (c_int, [engine_t, c_uint64, c_uint64, c_int, c_int]),
        "sortArrayAsync": (c_int, [engine_t, data_t, c_void_p]),
        "sortSynchronize": (c_int, [engine_t]),
        "sortPlanPasses": (c_int, [c_int, c_int, c_int, POINTER(c_int)]),
        "sortInjectFault": (c_int, [engine_t, c_int]),
        "sortEnableKernelTiming": (c_int, [engine_t, c_int]),
        "sortReadKernelTiming": (c_int, [engine_t, POINTER(ctypes.c_double), POINTER(c_int),
                                         POINTER(ctypes.c_double), POINTER(c_int)]),
        "sortArrayNoAlloc": (c_int, [data_t, c_void_p]),
        "sortSegmentedArray": (c_int, [engine_t, data_t, c_void_p, c_int, c_void_p]),
        "sortArrayTyped": (c_int, [engine_t, data_t, c_int, c_void_p]),
        "sortSelectKey": (c_int, [engine_t, data_t, c_int, POINTER(c_uint)]),
        "sortEnableGraphs": (c_int, [engine_t, c_int]),
        "sortGraphStats": (c_int, [engine_t, POINTER(c_int), POINTER(c_int)]),
        "sortServerCreate": (c_int, [POINTER(ServerConfig), POINTER(c_void_p)]),
        "sortServerSubmit": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                     c_void_p, c_void_p, POINTER(ctypes.c_ulonglong)]),
        "sortServerPoll": (c_int, [c_void_p, ctypes.c_ulonglong, POINTER(c_int)]),
        "sortServerWait": (c_int, [c_void_p, ctypes.c_ulonglong, POINTER(ctypes.c_double)]),
        "sortServerDestroy": (c_int, [c_void_p]),
        "bwtStatusString": (c_char_p, [c_int]),
        "bwtCreateEngine": (c_int, [c_char_p, POINTER(c_void_p)]),
        "bwtDestroyEngine": (c_int, [c_void_p]),
        "bwtSortBlock": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, POINTER(c_int),
                                 POINTER(c_int), POINTER(ctypes.c_float)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def sort_status_string(status: int) -> str | None:
    s = load_library().sortStatusString(int(status))
    return s.decode() if s is not None else None


class MgpuException(RuntimeError):
    """A non-success sortStatus_t (inc/mgpusort.hpp:12-20)."""

    def __init__(self, status: int):
        self.status = int(status)
        super().__init__(sort_status_string(status) or f"status {status}")


def check(status: int) -> None:
    if status != SortStatus.SUCCESS:
        raise MgpuException(status)


def plan_passes(first_bit: int, end_bit: int, bit_pass: int = 0) -> list[int]:
    """Digit widths of the passes a sort would run (sortPlanPasses)."""
    widths = (c_int * 32)()
    n = load_library().sortPlanPasses(first_bit, end_bit, bit_pass, widths)
    if n < 0:
        raise MgpuException(SortStatus.INVALID_VALUE)
    return list(widths[:n])


class MgpuSort:
    """Engine handle with reference counting (inc/mgpusort.hpp:83-114)."""

    def __init__(self, kernel_path: str = ""):
        lib = load_library()
        handle = c_void_p()
        check(lib.sortCreateEngine(kernel_path.encode(), ctypes.byref(handle)))
        self._engine = handle

    @property
    def handle(self) -> c_void_p:
        return self._engine

    def release(self) -> None:
        if self._engine:
            load_library().sortReleaseEngine(self._engine)
            self._engine = c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def sort_array(self, data: SortData) -> int:
        return load_library().sortArray(self._engine, ctypes.byref(data))

    def sort_array_ex(self, data: SortData, num_threads: int = 256,
                      values_per_thread: int = 8, bit_pass: int = 6,
                      use_trans_list: bool = False) -> int:
        return load_library().sortArrayEx(self._engine, ctypes.byref(data),
                                          num_threads, values_per_thread,
                                          bit_pass, use_trans_list)

    def sort_array_async(self, data: SortData, stream: int) -> int:
        return load_library().sortArrayAsync(self._engine, ctypes.byref(data),
                                             c_void_p(stream))

    def sort_array_typed(self, data: SortData, key_type: int, stream: int = 0) -> int:
        """sortArrayTyped: KEY_INT32 / KEY_FLOAT32 keys (KEY_UINT32 = plain)."""
        return load_library().sortArrayTyped(self._engine, ctypes.byref(data), int(key_type),
                                             c_void_p(stream))

    def select_key(self, data: SortData, k: int) -> tuple[int, int]:
        """sortSelectKey: (status, k-th smallest key after sorting data)."""
        v = c_uint(0)
        st = load_library().sortSelectKey(self._engine, ctypes.byref(data), int(k),
                                          ctypes.byref(v))
        return st, int(v.value)

    def enable_graphs(self, enable: bool) -> int:
        return load_library().sortEnableGraphs(self._engine, 1 if enable else 0)

    def graph_stats(self) -> tuple[int, int]:
        """(graph replays so far, graphs cached now)."""
        r, c = c_int(0), c_int(0)
        check(load_library().sortGraphStats(self._engine, ctypes.byref(r), ctypes.byref(c)))
        return r.value, c.value

    def synchronize(self) -> int:
        return load_library().sortSynchronize(self._engine)

    def sort_segmented(self, data: SortData, offsets_ptr: int, num_segments: int,
                       stream: int = 0) -> int:
        """sortSegmentedArray: offsets_ptr is a device int array of
        num_segments + 1 segment boundaries."""
        return load_library().sortSegmentedArray(self._engine, ctypes.byref(data),
                                                 c_void_p(offsets_ptr), num_segments,
                                                 c_void_p(stream))

    def enable_kernel_timing(self, enable: bool = True) -> None:
        check(load_library().sortEnableKernelTiming(self._engine, int(enable)))

    def read_kernel_timing(self) -> dict:
        """{'upsweep_ms', 'upsweep_launches', 'pass_ms', 'pass_launches'}
        summed since the last read (waits for the timed launches)."""
        um, pm = ctypes.c_double(), ctypes.c_double()
        ul, pl = c_int(), c_int()
        check(load_library().sortReadKernelTiming(self._engine, ctypes.byref(um),
                                                  ctypes.byref(ul), ctypes.byref(pm),
                                                  ctypes.byref(pl)))
        return {"upsweep_ms": um.value, "upsweep_launches": ul.value,
                "pass_ms": pm.value, "pass_launches": pl.value}

    def inject_fault(self, tile: int) -> int:
        return load_library().sortInjectFault(self._engine, tile)

    def sort_device(self, keys_ptr: int, values_ptr: int, n: int, num_bits: int) -> int:
        return load_library().sortDevice(self._engine, keys_ptr, values_ptr, n, num_bits)

    def sort_host(self, keys, values, num_bits: int) -> int:
        """keys / values: writable uint32 numpy arrays (values may be None)."""
        import numpy as np
        assert keys.dtype == np.uint32 and keys.flags.c_contiguous
        kp = keys.ctypes.data_as(POINTER(c_uint))
        vp = None
        if values is not None:
            assert values.dtype == np.uint32 and values.flags.c_contiguous
            vp = values.ctypes.data_as(POINTER(c_uint))
        return load_library().sortHost(self._engine, kp, vp, int(keys.size), num_bits)


def sort_array_no_alloc(data: SortData, stream: int = 0) -> int:
    """sortArrayNoAlloc: sortArray without an engine and without allocating;
    waits for the sort. For callers whose device memory is all pre-budgeted."""
    return load_library().sortArrayNoAlloc(ctypes.byref(data), c_void_p(stream))


class SortServer:
    """sortServer_t: submit host-memory sort requests, wait for tickets."""

    def __init__(self, memory_budget: int = 0, slots: int = 0, coalesce_max: int = 0,
                 max_batch_elements: int = 0, max_batch_requests: int = 0):
        cfg = ServerConfig(memory_budget, slots, coalesce_max, max_batch_elements,
                           max_batch_requests)
        h = c_void_p()
        check(load_library().sortServerCreate(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def submit(self, keys_ptr: int, values_ptr: int | None, n: int, first_bit: int,
               end_bit: int, keys_out_ptr: int, values_out_ptr: int | None) -> int:
        t = ctypes.c_ulonglong()
        check(load_library().sortServerSubmit(self._h, c_void_p(keys_ptr),
                                              c_void_p(values_ptr or 0), n, first_bit,
                                              end_bit, c_void_p(keys_out_ptr),
                                              c_void_p(values_out_ptr or 0),
                                              ctypes.byref(t)))
        return t.value

    def poll(self, ticket: int) -> bool:
        d = c_int()
        check(load_library().sortServerPoll(self._h, ticket, ctypes.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int) -> tuple[int, float]:
        """(status, seconds from submission to completion)"""
        lat = ctypes.c_double()
        st = load_library().sortServerWait(self._h, ticket, ctypes.byref(lat))
        return st, lat.value

    def close(self) -> None:
        if self._h:
            load_library().sortServerDestroy(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MgpuSortData(SortData):
    """sortData_d that remembers which buffers the caller attached, so that
    reset() frees only the library's own (inc/mgpusort.hpp:24-81)."""

    def __init__(self):
        super().__init__()
        self._attached_keys = [False, False]
        self._attached_vals = [[False, False] for _ in range(6)]

    def attach_key(self, ptr: int, i: int = 0) -> None:
        self.keys[i] = ptr
        self._attached_keys[i ^ self.parity] = True

    def attach_val(self, j: int, ptr: int, i: int = 0) -> None:
        self.values[j][i] = ptr
        self._attached_vals[j][i ^ self.parity] = True

    def alloc(self, engine: MgpuSort, max_elements: int, value_count: int) -> int:
        self.maxElements = max_elements
        self.numElements = max_elements
        self.valueCount = value_count
        return load_library().sortAllocData(engine.handle, ctypes.byref(self))

    def reset(self) -> None:
        for i in range(2):
            if self._attached_keys[i]:
                self.keys[i ^ self.parity] = 0
            for j in range(6):
                if self._attached_vals[j][i]:
                    self.values[j][i ^ self.parity] = 0
        load_library().sortFreeData(ctypes.byref(self))
        self._attached_keys = [False, False]
        self._attached_vals = [[False, False] for _ in range(6)]


class BwtStatus(enum.IntEnum):
    """bwtStatus_t, in the order of inc/mgpubwt.h:21-34."""
    SUCCESS = 0
    NOT_INITIALIZED = 1
    DEVICE_ALLOC_FAILED = 2
    INVALID_CONTEXT = 3
    KERNEL_NOT_FOUND = 4
    KERNEL_ERROR = 5
    LAUNCH_ERROR = 6
    INVALID_VALUE = 7
    DEVICE_ERROR = 8
    NOT_IMPLEMENTED = 9
    UNSUPPORTED_DEVICE = 10
    SORT_ERROR = 11


def bwt_status_string(status: int) -> str | None:
    s = load_library().bwtStatusString(int(status))
    return s.decode() if s is not None else None


class BwtEngine:
    """bwtCreateEngine / bwtSortBlock / bwtDestroyEngine (inc/mgpubwt.h)."""

    def __init__(self, kernel_path: str = ""):
        lib = load_library()
        handle = c_void_p()
        st = lib.bwtCreateEngine(kernel_path.encode(), ctypes.byref(handle))
        if st != BwtStatus.SUCCESS:
            raise RuntimeError(bwt_status_string(st) or f"status {st}")
        self._engine = handle

    def sort_block(self, block, key_size: int):
        """Returns (status, indices int32[n], transform uint8[n], segCount,
        avSegSize) for the bytes of `block` (bytes or a uint8 array)."""
        import numpy as np
        data = np.frombuffer(bytes(block), dtype=np.uint8) if not hasattr(block, "dtype") \
            else np.ascontiguousarray(block, dtype=np.uint8)
        n = int(data.size)
        indices = np.zeros(max(n, 1), dtype=np.int32)
        transform = np.zeros(max(n, 1), dtype=np.uint8)
        seg = c_int(-1)
        av = ctypes.c_float(-1.0)
        st = load_library().bwtSortBlock(
            self._engine, data.ctypes.data_as(c_void_p), n, int(key_size),
            transform.ctypes.data_as(c_void_p), indices.ctypes.data_as(POINTER(c_int)),
            ctypes.byref(seg), ctypes.byref(av))
        return int(st), indices[:n], transform[:n], seg.value, av.value

    def close(self) -> None:
        if self._engine:
            load_library().bwtDestroyEngine(self._engine)
            self._engine = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""CPU checks of the C ABI: the library loads, exports exactly what
include/*.h declares, and its host-only entry points behave like the
reference's (no device work is launched here)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import HAVE_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(?:SORTAPI|BWTAPI)\s+(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported_functions(path):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol(lib):
    from mgpu_old_b200 import api
    declared = declared_functions()
    reference = {"sortStatusString", "sortCreateEngine", "sortLoadKernel",
                 "sortIncEngine", "sortReleaseEngine", "sortCreateData",
                 "sortDestroyData", "sortAllocData", "sortFreeData", "sortArray",
                 "sortArrayEx", "sortHost", "sortDevice"}
    assert reference <= declared
    exported = exported_functions(api.LIB_PATH)
    assert declared == exported, (declared ^ exported)
    assert declared == set(api.EXPORTED_SYMBOLS)
    for name in declared:
        assert getattr(lib, name) is not None


def test_status_strings(lib):
    from mgpu_old_b200 import api
    for s in api.SortStatus:
        assert api.sort_status_string(s) == "SORT_STATUS_" + s.name
    assert api.sort_status_string(14) is None
    assert api.sort_status_string(-1) is None


def test_sortdata_layout(lib):
    from mgpu_old_b200 import api
    d = api.SortData
    assert ctypes.sizeof(d) == 144
    offs = {f[0]: getattr(d, f[0]).offset for f in d._fields_}
    assert offs == {"maxElements": 0, "numElements": 4, "valueCount": 8, "firstBit": 12,
                    "endBit": 16, "preserveEndKeys": 20, "earlyExit": 21, "parity": 24,
                    "keys": 32, "values": 48}


@pytest.mark.parametrize("bits", list(range(1, 33)))
def test_default_plan(lib, bits):
    from mgpu_old_b200 import api
    w = api.plan_passes(0, bits)
    assert sum(w) == bits
    assert len(w) == (bits + 7) // 8
    assert max(w) - min(w) <= 1 and max(w) <= 8


@pytest.mark.parametrize("bits", [1, 5, 6, 7, 18, 24, 31, 32])
@pytest.mark.parametrize("bit_pass", [1, 2, 3, 4, 5, 6])
def test_ex_plan_matches_reference(lib, oracle_mod, bits, bit_pass):
    """sortArrayEx's plan has the reference's pass count and widths
    (mgpusort.cpp:626-646), so parity after the sort matches the reference."""
    from mgpu_old_b200 import api
    ours = api.plan_passes(32 - bits, 32, bit_pass)
    ref = oracle_mod.reference_ex_plan(bits, bit_pass)
    assert sorted(ours) == sorted(ref)
    assert ours == ref  # narrow passes first, as the reference's table walk


def test_plan_rejects_bad_ranges(lib):
    from mgpu_old_b200 import api
    widths = (ctypes.c_int * 32)()
    assert lib.sortPlanPasses(-1, 8, 0, widths) == -1
    assert lib.sortPlanPasses(0, 33, 0, widths) == -1
    assert lib.sortPlanPasses(9, 8, 0, widths) == -1
    assert lib.sortPlanPasses(4, 4, 0, widths) == 0
    assert lib.sortPlanPasses(0, 8, 7, widths) == -1


def test_null_arguments_are_rejected(lib):
    from mgpu_old_b200 import api
    INVALID = api.SortStatus.INVALID_VALUE
    assert lib.sortArray(None, None) == INVALID
    assert lib.sortIncEngine(None) == INVALID
    assert lib.sortReleaseEngine(None) == api.SortStatus.SUCCESS
    assert lib.sortFreeData(None) == INVALID
    assert lib.sortDestroyData(None) == api.SortStatus.SUCCESS
    assert lib.sortSynchronize(None) == INVALID
    assert lib.sortCreateEngine(b"", None) == INVALID


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device error path")
def test_create_engine_without_a_device_fails_cleanly(lib):
    from mgpu_old_b200 import api
    h = ctypes.c_void_p()
    st = lib.sortCreateEngine(b"", ctypes.byref(h))
    assert st in (api.SortStatus.INVALID_CONTEXT, api.SortStatus.UNSUPPORTED_DEVICE)
    assert not h.value


def test_bwt_status_strings(lib):
    from mgpu_old_b200 import api
    for s in api.BwtStatus:
        assert api.bwt_status_string(s) == "BWT_STATUS_" + s.name
    assert api.bwt_status_string(12) is None
    assert api.bwt_status_string(-1) is None


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device error path")
def test_bwt_create_engine_without_gpu(lib):
    from mgpu_old_b200 import api
    handle = ctypes.c_void_p()
    st = lib.bwtCreateEngine(b"", ctypes.byref(handle))
    assert st != api.BwtStatus.SUCCESS
    assert not handle.value


def test_bwt_host_only_block_without_engine(lib, oracle_mod):
    """Blocks under 3000 bytes are sorted on the host; no engine is needed
    (mgpubwt.cpp:217-221)."""
    import numpy as np
    blk = np.frombuffer(b"abracadabra", dtype=np.uint8).copy()
    idx = (ctypes.c_int * 11)()
    xf = (ctypes.c_ubyte * 11)()
    seg, av = ctypes.c_int(), ctypes.c_float()
    st = lib.bwtSortBlock(None, blk.ctypes.data_as(ctypes.c_void_p), 11, 4, xf, idx,
                          ctypes.byref(seg), ctypes.byref(av))
    assert st == 0
    assert bytes(xf) == b"rdarcaaaabb"
    e_idx, _, e_seg, e_av = oracle_mod.bwt(blk, 4)
    assert list(idx) == list(e_idx) and seg.value == e_seg and av.value == e_av

"""Parity at the benchmark configurations' own sizes and seeds, bit for bit
against the oracle, through the C ABI.

  * keys_u32_1M: 1,048,576 uniform 32-bit keys, bits [0, 32), keys only;
    checked against the oracle's std::stable_sort and its LSD restatement of
    sort/src/cpusort/cpusort.cpp:122-186.
  * pairs_and24_32M: 33,554,432 keys = (r1 & r2) & 0xFFFFFF, value = index,
    bits [0, 24).
  * multi6_17bit_16M: 16,777,216 keys uniform in [0, 2^17) with six random
    value arrays, bits [0, 32).
  * pairs_u32_64M: 67,108,864 uniform 32-bit keys, value = index, bits [0, 32).
  * keys_u32_64M: 67,108,864 uniform 32-bit keys, keys only (the keys-only
    passes of at least 40 Mi keys run their own tile shape).
  * segments_10k: 10,000 lognormal segments (median 2048, sigma 2) through
    sortSegmentedArray, against one stable sort per segment; also the same
    sizes rescaled to 2^26 pairs in total.

Inputs come from mgpu_old_b200.workloads, the generators the benchmark uses.
Tolerance: exact (every key and every value array)."""
import os

import numpy as np
import pytest

from sortcase import DeviceSort

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _widths(first_bit, end_bit):
    bits = end_bit - first_bit
    p = (bits + 7) // 8
    return [bits // p + (i < bits % p) for i in range(p)]


def _sort_and_compare(engine, case, oracle_mod, also_stable=False):
    import torch
    from mgpu_old_b200 import api
    ds = DeviceSort(case.keys, case.values, case.value_count, case.first_bit, case.end_bit)
    torch.cuda.synchronize()
    st = engine.sort_array(ds.data)
    assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
    st = engine.synchronize()
    assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
    keys, vals = ds.result()
    del ds
    torch.cuda.empty_cache()
    ek, ev = oracle_mod.sort_lsd(case.keys, case.values, case.value_count, case.first_bit,
                                 _widths(case.first_bit, case.end_bit), 1 << 15, THREADS)
    assert np.array_equal(keys, ek), "keys differ from the oracle"
    assert len(vals) == len(ev)
    for i, (a, b) in enumerate(zip(vals, ev)):
        assert np.array_equal(a, b), f"value array {i} differs from the oracle"
    if also_stable:
        sk, sv = oracle_mod.sort_stable(case.keys, case.values, case.value_count,
                                        case.first_bit, case.end_bit)
        assert np.array_equal(keys, sk)
        for a, b in zip(vals, sv):
            assert np.array_equal(a, b)


def test_keys_u32_1m(engine, oracle_mod):
    from mgpu_old_b200 import workloads
    case = workloads.keys_uniform32()
    assert case.n == 1_048_576
    _sort_and_compare(engine, case, oracle_mod, also_stable=True)
    # The reference's own CPU sort (cpusort.cpp Sort2: eight blocked 4-bit
    # passes), built from its source, gives the same keys.
    ref = oracle_mod.ref_lib()
    if ref is not None:
        k = np.array(case.keys, copy=True)
        ref.ref_cpusort_sort2(oracle_mod._p(k), k.size, 2048)
        assert np.array_equal(k, np.sort(case.keys))


def test_pairs_and24_32m(engine, oracle_mod):
    from mgpu_old_b200 import workloads
    case = workloads.pairs_and24()
    assert case.n == 33_554_432 and (case.first_bit, case.end_bit) == (0, 24)
    _sort_and_compare(engine, case, oracle_mod)


def test_multi6_17bit_16m_six_value_arrays(engine, oracle_mod):
    from mgpu_old_b200 import workloads
    case = workloads.multi6_17bit()
    assert case.n == 16_777_216 and case.value_count == 6
    _sort_and_compare(engine, case, oracle_mod)


def test_pairs_u32_64m(engine, oracle_mod):
    from mgpu_old_b200 import workloads
    case = workloads.pairs_uniform32()
    assert case.n == 67_108_864
    _sort_and_compare(engine, case, oracle_mod)


def test_keys_u32_64m(engine, oracle_mod):
    # Keys only from 40 Mi keys on: the large-array tile class.
    from mgpu_old_b200 import workloads
    case = workloads.keys_uniform32_64m()
    assert case.n == 67_108_864 and case.value_count == 0
    _sort_and_compare(engine, case, oracle_mod)


@pytest.mark.parametrize("scale_to", [None, 1 << 26], ids=["unscaled", "total_64M"])
def test_segments_10k_lognormal(engine, oracle_mod, scale_to):
    import torch
    from mgpu_old_b200 import api, workloads
    case = workloads.segments_lognormal(scale_to=scale_to)
    assert case.num_segments == 10_000
    if scale_to:
        # Rescaled sizes are rounded per segment: the total is within a few of 2^26.
        assert abs(int(case.offsets[-1]) - scale_to) < 100
    ds = DeviceSort(case.keys, case.values, case.value_count, case.first_bit, case.end_bit)
    offs = torch.from_numpy(case.offsets.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    st = engine.sort_segmented(ds.data, offs.data_ptr(), case.num_segments)
    assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
    assert engine.synchronize() == api.SortStatus.SUCCESS
    keys, (vals,) = ds.result()
    del ds
    torch.cuda.empty_cache()
    ek, (ev,) = oracle_mod.sort_segments(case.keys, case.values, case.value_count,
                                         case.offsets, case.first_bit, case.end_bit)
    assert np.array_equal(keys, ek)
    assert np.array_equal(vals, ev)

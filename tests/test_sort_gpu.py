"""Parity of the CUDA path with the oracle, through the C ABI (sortArray,
sortArrayEx, sortHost, sortDevice). Bit-exact: this is integer work."""
import glob
import os

import numpy as np
import pytest

from sortcase import DeviceSort, check_index_result, run_sort, to_dev

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def rand_u32(rng, n, high=1 << 32):
    return rng.integers(0, high, n, dtype=np.uint64).astype(np.uint32)


def expect(oracle_mod, keys, vals, vc, fb, eb):
    return oracle_mod.sort_stable(keys, vals, vc, fb, eb)


def assert_same(ds, ek, ev):
    k, v = ds.result()
    assert np.array_equal(k, ek), f"keys differ at {np.flatnonzero(k != ek)[:8]}"
    for i, (a, b) in enumerate(zip(v, ev)):
        assert np.array_equal(a, b), f"values{i + 1} differ at {np.flatnonzero(a != b)[:8]}"


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f) for f in FIXTURES])
def test_golden_fixtures(engine, path):
    z = np.load(path)
    vc = int(z["value_count"])
    arrays = 1 if vc == -1 else vc
    vals = [z[f"values{i}"] for i in range(vc)] if vc > 0 else []
    ds = run_sort(engine, z["keys"], vals, vc, int(z["first_bit"]), int(z["end_bit"]))
    assert_same(ds, z["expect_keys"], [z[f"expect_values{i}"] for i in range(arrays)])


# Around the tile sizes of the sort kernel with the shipped tile shapes
# (7168 keys only, 7680 indices or one value array, 6144 several value
# arrays), two tiles, and of other shapes the autotuner may pick (5120).
SIZES = [1, 2, 31, 255, 4095, 4097, 5119, 5120, 5121, 6143, 6144, 6145, 7167, 7168,
         7169, 7679, 7680, 7681, 10241, 12289, 15361, 100003]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("vc", [-1, 0, 1, 2, 3, 4, 5, 6])
def test_value_modes_and_sizes(engine, oracle_mod, n, vc):
    rng = np.random.Generator(np.random.MT19937(n * 8 + vc + 1))
    keys = rand_u32(rng, n)
    keys[: n // 3] &= np.uint32(0x00FF00FF)   # ties and skew
    vals = [rand_u32(rng, n) for _ in range(max(vc, 0))]
    ds = run_sort(engine, keys, vals, vc, 0, 32)
    assert_same(ds, *expect(oracle_mod, keys, vals, vc, 0, 32))


RANGES = [(0, 32), (0, 24), (7, 25), (16, 32), (31, 32), (0, 1), (3, 4), (0, 8),
          (8, 16), (5, 29), (1, 31), (12, 13), (0, 9), (20, 32)]


@pytest.mark.parametrize("fb,eb", RANGES)
@pytest.mark.parametrize("vc", [0, 1, -1])
def test_bit_ranges(engine, oracle_mod, fb, eb, vc):
    rng = np.random.Generator(np.random.MT19937(fb * 64 + eb))
    n = 20000 + fb * 131
    keys = rand_u32(rng, n)
    keys[::2] &= np.uint32(0x0F0F0F0F)
    vals = [np.arange(n, dtype=np.uint32)] if vc == 1 else []
    ds = run_sort(engine, keys, vals, vc, fb, eb)
    ek, ev = expect(oracle_mod, keys, vals, vc, fb, eb)
    assert_same(ds, ek, ev)
    from mgpu_old_b200 import api
    assert ds.data.parity == len(api.plan_passes(fb, eb)) % 2


@pytest.mark.parametrize("bit_pass", [1, 2, 3, 4, 5, 6, 0, 9])
@pytest.mark.parametrize("vc", [0, 2])
def test_sort_array_ex(engine, oracle_mod, bit_pass, vc):
    from mgpu_old_b200 import api
    rng = np.random.Generator(np.random.MT19937(bit_pass + 100 * vc))
    n = 30001
    keys = rand_u32(rng, n, 1 << 26) << np.uint32(3)
    vals = [rand_u32(rng, n) for _ in range(vc)]
    fb, eb = 3, 29
    ds = run_sort(engine, keys, vals, vc, fb, eb, how="ex", bit_pass=bit_pass)
    assert_same(ds, *expect(oracle_mod, keys, vals, vc, fb, eb))
    ref_passes = len(oracle_mod.reference_ex_plan(eb - fb, bit_pass))
    assert ds.data.parity == ref_passes % 2


def test_sort_array_ex_rejects_bad_config(engine):
    from mgpu_old_b200 import api
    ds = DeviceSort(np.arange(10, dtype=np.uint32), [], 0, 0, 32)
    assert engine.sort_array_ex(ds.data, 64, 8, 4) == api.SortStatus.INVALID_VALUE
    assert engine.sort_array_ex(ds.data, 128, 4, 4) == api.SortStatus.INVALID_VALUE


def test_swaps_and_parity(engine, oracle_mod):
    """After the sort keys[0] holds the result; buffers were swapped once per
    pass, so the caller's original buffer is at [parity]."""
    rng = np.random.Generator(np.random.MT19937(7))
    keys = rand_u32(rng, 5000)
    for fb, eb, passes in [(0, 32, 4), (0, 24, 3), (0, 8, 1), (0, 16, 2)]:
        ds = run_sort(engine, keys, [np.arange(5000, dtype=np.uint32)], 1, fb, eb)
        assert ds.data.parity == passes % 2
        assert ds.data.keys[ds.data.parity] == ds.original_keys_ptr
        ek, ev = expect(oracle_mod, keys, [np.arange(5000, dtype=np.uint32)], 1, fb, eb)
        assert_same(ds, ek, ev)


def test_nothing_past_num_elements_is_written(engine):
    n = 3000
    rng = np.random.Generator(np.random.MT19937(8))
    keys = rand_u32(rng, n)
    ds = run_sort(engine, keys, [rand_u32(rng, n)], 1, 0, 32)
    for ptr in (ds.data.keys[0], ds.data.keys[1], ds.data.values[0][0],
                ds.data.values[0][1]):
        tail = ds.read_full(ptr)[n:]
        assert (tail == 0xFFFFFFFF).all()   # the fill of to_dev, untouched


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_unaligned_buffers(engine, oracle_mod, offset):
    """Buffers that are not 16-byte aligned take the plain-load path."""
    rng = np.random.Generator(np.random.MT19937(offset))
    n = 50000
    keys = rand_u32(rng, n)
    vals = [rand_u32(rng, n), rand_u32(rng, n)]
    ds = run_sort(engine, keys, vals, 2, 0, 32, offset=offset)
    assert_same(ds, *expect(oracle_mod, keys, vals, 2, 0, 32))


def test_early_exit_skips_single_digit_passes(engine, oracle_mod):
    rng = np.random.Generator(np.random.MT19937(9))
    n = 40000
    keys = (rand_u32(rng, n, 1 << 16) << np.uint32(8)) | np.uint32(0x5A0000A5 & 0xFF0000FF)
    ek, ev = expect(oracle_mod, keys, [], -1, 0, 32)
    ds = run_sort(engine, keys, [], -1, 0, 32, early_exit=True)
    assert_same(ds, ek, ev)
    assert ds.data.parity == 0            # 2 of 4 passes run
    ds = run_sort(engine, keys, [], -1, 0, 32, early_exit=False)
    assert_same(ds, ek, ev)               # same result with all 4 passes


def test_early_exit_all_passes_skipped_index_mode(engine):
    n = 10000
    keys = np.full(n, 0x12345678, np.uint32)
    ds = run_sort(engine, keys, [], -1, 0, 32, early_exit=True)
    k, (v,) = ds.result()
    assert ds.data.parity == 0
    assert np.array_equal(k, keys)
    assert np.array_equal(v, np.arange(n, dtype=np.uint32))


def test_presorted_and_reverse(engine, oracle_mod):
    n = 70000
    for keys in (np.arange(n, dtype=np.uint32) * np.uint32(977),
                 (np.arange(n, dtype=np.uint32) * np.uint32(977))[::-1].copy()):
        ds = run_sort(engine, keys, [], -1, 0, 32)
        k, (v,) = ds.result()
        check_index_result(keys, 0, 32, k, v)


def test_invalid_arguments(engine):
    from mgpu_old_b200 import api
    INVALID = api.SortStatus.INVALID_VALUE
    keys = np.arange(100, dtype=np.uint32)
    ds = DeviceSort(keys, [], 0, 0, 32)
    d = ds.data
    d.numElements = d.maxElements + 1
    assert engine.sort_array(d) == INVALID
    d.numElements = 100
    d.firstBit, d.endBit = 0, 33
    assert engine.sort_array(d) == INVALID
    d.firstBit, d.endBit = -1, 8
    assert engine.sort_array(d) == INVALID
    d.firstBit, d.endBit = 9, 9
    assert engine.sort_array(d) == api.SortStatus.SUCCESS   # nothing to do
    d.firstBit, d.endBit = 0, 32
    d.valueCount = 7
    assert engine.sort_array(d) == INVALID
    d.valueCount = 1                                        # values1 missing
    assert engine.sort_array(d) == INVALID
    d.valueCount = 0
    d.numElements = 0
    assert engine.sort_array(d) == api.SortStatus.SUCCESS
    assert d.parity == 0


def test_sort_host(engine, oracle_mod):
    rng = np.random.Generator(np.random.MT19937(11))
    n = 123457
    keys = rand_u32(rng, n)
    vals = np.arange(n, dtype=np.uint32)
    ek, (ev,) = expect(oracle_mod, keys, [vals], 1, 0, 24)
    k, v = keys.copy(), vals.copy()
    assert engine.sort_host(k, v, 24) == 0
    assert np.array_equal(k, ek) and np.array_equal(v, ev)
    k = keys.copy()
    assert engine.sort_host(k, None, 32) == 0
    assert np.array_equal(k, np.sort(keys))


@pytest.mark.parametrize("bits", [32, 24, 8, 13])
def test_sort_device_result_lands_in_callers_buffers(engine, oracle_mod, bits):
    import torch
    rng = np.random.Generator(np.random.MT19937(bits))
    n = 77777
    keys = rand_u32(rng, n)
    vals = np.arange(n, dtype=np.uint32)
    kt, kp = to_dev(keys, n)
    vt, vp = to_dev(vals, n)
    torch.cuda.synchronize()
    assert engine.sort_device(kp, vp, n, bits) == 0
    ek, (ev,) = expect(oracle_mod, keys, [vals], 1, 0, bits)
    assert np.array_equal(kt.cpu().numpy().view(np.uint32), ek)
    assert np.array_equal(vt.cpu().numpy().view(np.uint32), ev)


def test_library_managed_data(engine, lib, oracle_mod):
    """sortCreateData / sortDestroyData and MgpuSortData attach semantics."""
    import ctypes
    import torch
    from mgpu_old_b200 import api
    p = ctypes.POINTER(api.SortData)()
    assert lib.sortCreateData(engine.handle, 5000, 2, ctypes.byref(p)) == 0
    d = p.contents
    assert d.maxElements == 6144 and d.numElements == 5000
    assert d.firstBit == 0 and d.endBit == 32 and d.valueCount == 2
    assert all(d.keys[i] for i in range(2))
    assert all(d.values[j][i] for j in range(2) for i in range(2))
    assert not any(d.values[j][i] for j in range(2, 6) for i in range(2))
    assert lib.sortDestroyData(p) == 0

    n = 9000
    rng = np.random.Generator(np.random.MT19937(12))
    keys = rand_u32(rng, n)
    kt, kp = to_dev(keys, n)
    sd = api.MgpuSortData()
    sd.attach_key(kp)
    assert sd.alloc(engine, n, -1) == 0
    sd.firstBit, sd.endBit = 0, 32          # Alloc leaves the bit range to the caller
    assert sd.keys[0] == kp and sd.keys[1] and sd.values[0][0] and sd.values[0][1]
    torch.cuda.synchronize()
    assert engine.sort_array(sd) == 0
    assert engine.synchronize() == 0
    ek, (ev,) = expect(oracle_mod, keys, [], -1, 0, 32)
    assert sd.parity == 0 and sd.keys[0] == kp     # four passes: back in place
    assert np.array_equal(kt.cpu().numpy().view(np.uint32), ek)
    sd.reset()                       # frees only the library's buffers
    assert sd.keys[0] == 0 and sd.keys[1] == 0
    torch.cuda.synchronize()
    assert kt.cpu().numpy().size == n   # the caller's buffer is still alive


def test_repeated_sorts_reuse_engine_state(engine, oracle_mod):
    """Scratch is self-cleaning between sorts of different shapes."""
    rng = np.random.Generator(np.random.MT19937(13))
    for n, vc, fb, eb in [(100000, 1, 0, 32), (5000, 0, 4, 20), (300000, 3, 0, 32),
                          (4096, -1, 0, 17), (100000, 1, 0, 32)]:
        keys = rand_u32(rng, n)
        vals = [rand_u32(rng, n) for _ in range(max(vc, 0))]
        ds = run_sort(engine, keys, vals, vc, fb, eb)
        assert_same(ds, *expect(oracle_mod, keys, vals, vc, fb, eb))


def test_two_engines(lib, oracle_mod):
    from mgpu_old_b200 import api
    import torch
    torch.zeros(1, device="cuda")
    e1, e2 = api.MgpuSort(), api.MgpuSort()
    assert lib.sortIncEngine(e1.handle) == 0
    assert lib.sortReleaseEngine(e1.handle) == 0
    rng = np.random.Generator(np.random.MT19937(14))
    keys = rand_u32(rng, 20000)
    for e in (e1, e2):
        ds = run_sort(e, keys, [], -1, 0, 32)
        assert_same(ds, *expect(oracle_mod, keys, [], -1, 0, 32))
    e1.release()
    e2.release()


def test_async_stream(engine, oracle_mod):
    import torch
    rng = np.random.Generator(np.random.MT19937(15))
    n = 200000
    keys = rand_u32(rng, n)
    ds = DeviceSort(keys, [np.arange(n, dtype=np.uint32)], 1, 0, 32)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    assert engine.sort_array_async(ds.data, s.cuda_stream) == 0
    assert engine.synchronize() == 0
    assert_same(ds, *expect(oracle_mod, keys, [np.arange(n, dtype=np.uint32)], 1, 0, 32))


def test_bounded_wait_reports_kernel_error(engine, oracle_mod):
    """A CTA that waits on a barrier nothing completes runs its bounded wait
    out: the sort reports KERNEL_ERROR (no fault, no hang) and the engine
    keeps working."""
    from mgpu_old_b200 import api
    import time
    import torch
    n = 3 * 4096
    keys = np.arange(n, dtype=np.uint32)[::-1].copy()
    ds = DeviceSort(keys, [], 0, 0, 32)
    torch.cuda.synchronize()
    assert engine.inject_fault(1) == 0
    t0 = time.time()
    assert engine.sort_array(ds.data) == 0
    assert engine.synchronize() == api.SortStatus.KERNEL_ERROR
    assert time.time() - t0 < 20
    rng = np.random.Generator(np.random.MT19937(16))
    keys = rand_u32(rng, 50000)
    ds = run_sort(engine, keys, [], -1, 0, 32)
    assert_same(ds, *expect(oracle_mod, keys, [], -1, 0, 32))

"""Batched segmented sort (sortSegmentedArray) against the oracle: each
segment sorted on its own, as one sortArray call per segment would. Bit-exact."""
import numpy as np
import pytest

from sortcase import DeviceSort, to_dev

pytestmark = pytest.mark.gpu


def rand_u32(rng, n, high=1 << 32):
    return rng.integers(0, high, n, dtype=np.uint64).astype(np.uint32)


def run_segmented(engine, keys, vals, vc, offsets, fb=0, eb=32):
    import torch
    from mgpu_old_b200 import api
    ds = DeviceSort(keys, vals, vc, fb, eb)
    offs_t, offs_p = to_dev(np.asarray(offsets, np.int32).view(np.uint32), offsets.size)
    torch.cuda.synchronize()
    st = engine.sort_segmented(ds.data, offs_p, offsets.size - 1)
    assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
    st = engine.synchronize()
    torch.cuda.synchronize()
    return ds, st


def layout(rng, sizes):
    offsets = np.zeros(len(sizes) + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    return offsets.astype(np.int32)


LAYOUTS = {
    "edges": [0, 1, 2, 511, 512, 513, 1023, 1024, 1025, 2047, 2048, 2049, 4095, 4096,
              4097, 0, 5119, 5120, 5121, 6143, 6144, 6145, 7167, 7168, 7169, 7680, 7681,
              15361, 30000, 100003, 3],
    "one_big": [250_001],
    "many_tiny": [int(x) for x in np.random.default_rng(1).integers(0, 40, 3000)],
    "lognormal": [int(x) for x in np.clip(np.rint(
        np.random.default_rng(2).lognormal(np.log(2048), 2.0, 400)), 1, 300_000)],
}


@pytest.mark.parametrize("name", sorted(LAYOUTS))
@pytest.mark.parametrize("vc", [1, 0, -1, 3])
def test_segmented_matches_oracle(engine, oracle_mod, name, vc):
    from mgpu_old_b200 import api
    rng = np.random.Generator(np.random.MT19937(len(name) * 10 + vc))
    offsets = layout(rng, LAYOUTS[name])
    n = int(offsets[-1])
    keys = rand_u32(rng, n)
    keys[::3] &= np.uint32(0x00FF00FF)
    vals = [rand_u32(rng, n) for _ in range(max(vc, 0))]
    ds, st = run_segmented(engine, keys, vals, vc, offsets)
    assert st == api.SortStatus.SUCCESS
    ek, ev = oracle_mod.sort_segments(keys, vals, vc, offsets, 0, 32)
    k, v = ds.result()
    assert np.array_equal(k, ek), np.flatnonzero(k != ek)[:10]
    for a, b in zip(v, ev):
        assert np.array_equal(a, b), np.flatnonzero(a != b)[:10]
    assert ds.data.parity == 0            # four passes over 32 bits


@pytest.mark.parametrize("fb,eb", [(0, 24), (7, 25), (31, 32)])
def test_segmented_bit_ranges(engine, oracle_mod, fb, eb):
    rng = np.random.Generator(np.random.MT19937(fb + eb))
    offsets = layout(rng, LAYOUTS["edges"])
    n = int(offsets[-1])
    keys = rand_u32(rng, n)
    vals = [np.arange(n, dtype=np.uint32)]
    ds, st = run_segmented(engine, keys, vals, 1, offsets, fb, eb)
    assert st == 0
    ek, ev = oracle_mod.sort_segments(keys, vals, 1, offsets, fb, eb)
    k, v = ds.result()
    assert np.array_equal(k, ek) and np.array_equal(v[0], ev[0])


def test_segmented_equals_sort_array_per_segment(engine):
    """The batched result equals separate sortArray calls on each segment."""
    from sortcase import run_sort
    rng = np.random.Generator(np.random.MT19937(77))
    sizes = [3, 600, 5000, 20000]
    offsets = layout(rng, sizes)
    n = int(offsets[-1])
    keys = rand_u32(rng, n)
    local = np.concatenate([np.arange(s, dtype=np.uint32) for s in sizes])
    ds, st = run_segmented(engine, keys, [local], 1, offsets)
    assert st == 0
    k, (v,) = ds.result()
    for i, s in enumerate(sizes):
        b, e = offsets[i], offsets[i + 1]
        one = run_sort(engine, keys[b:e], [local[b:e]], 1, 0, 32)
        k1, (v1,) = one.result()
        assert np.array_equal(k[b:e], k1) and np.array_equal(v[b:e], v1)


def test_segmented_rejects_bad_offsets(engine):
    """Offsets that do not cover [0, n) are reported as a device error and
    the engine keeps working."""
    from mgpu_old_b200 import api
    rng = np.random.Generator(np.random.MT19937(5))
    keys = rand_u32(rng, 1000)
    bad = np.array([0, 600, 400, 1000], np.int32)      # decreasing
    ds, st = run_segmented(engine, keys, [], 0, bad)
    assert st == api.SortStatus.KERNEL_ERROR
    short = np.array([0, 500, 900], np.int32)          # does not end at n
    ds, st = run_segmented(engine, keys, [], 0, short)
    assert st == api.SortStatus.KERNEL_ERROR
    good = np.array([0, 1000], np.int32)
    ds, st = run_segmented(engine, keys, [], 0, good)
    assert st == 0
    assert np.array_equal(ds.result()[0], np.sort(keys))

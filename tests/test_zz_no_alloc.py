"""sortArrayNoAlloc, the entry point for callers that cannot allocate device
memory (programs that pre-budget all of a GPU's memory for their own
allocator, or latency-critical loops where cudaMalloc/cudaFree would stall the
device), checked against sortArray through the C ABI: bit-exact, two calls in
a row on the shared static scratch. This file sorts last on purpose."""
import numpy as np
import pytest

from sortcase import DeviceSort

pytestmark = pytest.mark.gpu


def _rand(rng, n, high=1 << 32):
    return rng.integers(0, high, n, dtype=np.uint64).astype(np.uint32)


CASES = [
    # (n, valueCount, firstBit, endBit, seed)
    (1_000_003, 1, 0, 32, 1),
    (4_194_304, 3, 5, 29, 2),    # the maximum size, three value arrays
]


def test_no_alloc_matches_sort_array_two_calls_in_a_row(engine):
    import torch
    from mgpu_old_b200 import api
    for n, vc, fb, eb, seed in CASES:
        rng = np.random.Generator(np.random.MT19937(seed))
        keys = _rand(rng, n)
        keys[::5] &= np.uint32(0x00FFFF00)       # ties, skewed digits
        vals = [_rand(rng, n) for _ in range(vc)]
        ref = DeviceSort(keys, vals, vc, fb, eb)
        mine = DeviceSort(keys, vals, vc, fb, eb)
        torch.cuda.synchronize()
        assert engine.sort_array(ref.data) == api.SortStatus.SUCCESS
        assert engine.synchronize() == api.SortStatus.SUCCESS
        st = api.sort_array_no_alloc(mine.data, 0)
        assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
        torch.cuda.synchronize()
        assert mine.data.parity == ref.data.parity
        rk, rv = ref.result()
        mk, mv = mine.result()
        assert np.array_equal(mk, rk)
        for a, b in zip(mv, rv):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("n,vc,fb,eb,offset,seed", [
    (300_001, 1, 3, 9, 0, 4),      # one narrow pass
    (250_007, 2, 0, 32, 1, 5),     # buffers 4 bytes past a 16-byte boundary: plain loads
    (4_096, -1, 7, 25, 3, 6),      # index mode, unaligned, one tile
])
def test_no_alloc_against_oracle(engine, oracle_mod, n, vc, fb, eb, offset, seed):
    """Bit-exact against the CPU oracle (std::stable_sort by the bit field),
    twice in a row, including the path with plain loads for buffers that
    are not 16-byte aligned."""
    import torch
    from mgpu_old_b200 import api
    rng = np.random.Generator(np.random.MT19937(seed))
    keys = _rand(rng, n)
    keys[::3] &= np.uint32(0x0000FFF0)
    vals = [_rand(rng, n) for _ in range(max(vc, 0))]
    ek, ev = oracle_mod.sort_stable(keys, vals, vc, fb, eb)
    for _ in range(2):
        ds = DeviceSort(keys, vals, vc, fb, eb, offset=offset)
        torch.cuda.synchronize()
        st = api.sort_array_no_alloc(ds.data, 0)
        assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
        mk, mv = ds.result()
        assert np.array_equal(mk, ek)
        for a, b in zip(mv, ev):
            assert np.array_equal(a, b)


def test_no_alloc_index_mode_and_size_limit(engine):
    import torch
    from mgpu_old_b200 import api
    rng = np.random.Generator(np.random.MT19937(3))
    n = 777_777
    keys = _rand(rng, n, 1 << 20)
    ref = DeviceSort(keys, [], -1, 0, 20)
    mine = DeviceSort(keys, [], -1, 0, 20)
    torch.cuda.synchronize()
    assert engine.sort_array(ref.data) == 0 and engine.synchronize() == 0
    assert api.sort_array_no_alloc(mine.data, 0) == 0
    rk, (rv,) = ref.result()
    mk, (mv,) = mine.result()
    assert np.array_equal(mk, rk) and np.array_equal(mv, rv)

    big = api.NOALLOC_MAX_ELEMENTS + 1
    over = DeviceSort(np.zeros(big, np.uint32), [], 0, 0, 32)
    torch.cuda.synchronize()
    assert api.sort_array_no_alloc(over.data, 0) == api.SortStatus.CONFIG_NOT_SUPPORTED
    assert over.data.parity == 0

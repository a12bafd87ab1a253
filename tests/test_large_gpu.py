"""Maximum-size sorts, checked on the device through size-independent
properties (the oracle cannot hold them in seconds): 2^30 + 12345 keys with
generated indices (index mode) and 2^29 + 999 key-value pairs. The result
must be ordered by the bit field, the index/value array must be a
permutation that gathers the input keys into the output, and equal fields
must keep input order (tolerance: exact)."""
import pytest

from mgpu_old_b200 import api

pytestmark = pytest.mark.gpu


def device_data(n, value_count, first, end, torch):
    cap = (n + 2047) // 2048 * 2048
    g = torch.Generator(device="cuda").manual_seed(n)
    keys = torch.randint(-2 ** 31, 2 ** 31, (cap,), dtype=torch.int32, device="cuda",
                         generator=g)
    bufs = [keys, torch.empty_like(keys)]
    d = api.SortData()
    d.maxElements, d.numElements, d.valueCount = cap, n, value_count
    d.firstBit, d.endBit = first, end
    d.keys[0], d.keys[1] = keys.data_ptr(), bufs[1].data_ptr()
    vals = []
    if value_count != 0:
        v0 = torch.arange(cap, dtype=torch.int32, device="cuda")
        vals = [v0, torch.empty_like(v0)]
        d.values[0][0], d.values[0][1] = vals[0].data_ptr(), vals[1].data_ptr()
    src = keys[:n].clone()
    return d, bufs + vals, src


def check(d, tensors, src, first, end, torch):
    by_ptr = {t.data_ptr(): t for t in tensors}
    n = d.numElements
    out = by_ptr[d.keys[0]][:n]
    idx = by_ptr[d.values[0][0]][:n].to(torch.int64)
    u = out.to(torch.int64) & 0xFFFFFFFF
    mask = (1 << (end - first)) - 1
    field = (u >> first) & mask
    assert bool((field[1:] >= field[:-1]).all())
    # idx is a permutation of [0, n) ...
    seen = torch.zeros(n, dtype=torch.int32, device="cuda")
    seen.index_fill_(0, idx, 1)
    assert bool((idx >= 0).all()) and bool((idx < n).all()) and int(seen.sum()) == n
    # ... that gathers the input keys into the output, stably.
    assert bool((src[idx] == out).all())
    eq = field[1:] == field[:-1]
    assert bool((idx[1:][eq] > idx[:-1][eq]).all())


@pytest.mark.parametrize("n,value_count,first,end", [
    (2 ** 30 + 12345, -1, 0, 32),
    (2 ** 29 + 999, 1, 5, 27),
])
def test_maximum_size_sort(engine, n, value_count, first, end):
    import torch
    free, _ = torch.cuda.mem_get_info()
    if free < 64 * n + (8 << 30):
        pytest.skip("not enough device memory")
    d, tensors, src = device_data(n, value_count, first, end, torch)
    torch.cuda.synchronize()
    assert engine.sort_array(d) == 0
    assert engine.synchronize() == 0
    torch.cuda.synchronize()
    check(d, tensors, src, first, end, torch)
    del tensors, src
    torch.cuda.empty_cache()


def _tile_config(name):
    import os
    import re
    path = os.path.join(os.path.dirname(__file__), "..", "mgpu_old_b200", "csrc", "tile_config.h")
    with open(path) as f:
        return int(re.search(rf"#define {name} (\d+)", f.read()).group(1))


LARGE = _tile_config("MGPU_SORT_SINGLE_LARGE_ELEMENTS")


@pytest.mark.parametrize("n", [LARGE - 1, LARGE, LARGE + 7681])
@pytest.mark.parametrize("value_count,first,end", [(-1, 0, 32), (1, 0, 32), (1, 3, 20)])
def test_single_class_size_dispatch(engine, n, value_count, first, end):
    """sortArray with indices or one value array switches ranking kernels at
    MGPU_SORT_SINGLE_LARGE_ELEMENTS keys; both sides of the switch give the
    stable sort (exact)."""
    import torch
    d, tensors, src = device_data(n, value_count, first, end, torch)
    torch.cuda.synchronize()
    assert engine.sort_array(d) == 0
    assert engine.synchronize() == 0
    torch.cuda.synchronize()
    check(d, tensors, src, first, end, torch)
    del tensors, src
    torch.cuda.empty_cache()

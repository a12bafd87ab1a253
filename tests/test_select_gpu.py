"""The sort-based selection of the reference's select benchmark
(select/src/selecttest/mgpusorttest.cpp:3-32) through sortSelectKey: the k-th
smallest key equals numpy's (tolerance: exact)."""
import numpy as np
import pytest

from mgpu_old_b200 import api
from sortcase import DeviceSort

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 4097, 1 << 20])
def test_select_kth_key(engine, n):
    import torch
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    ref = np.sort(keys)
    for k in sorted({0, n // 3, n // 2, n - 1}):
        ds = DeviceSort(keys, [], 0, 0, 32)
        torch.cuda.synchronize()
        st, v = engine.select_key(ds.data, k)
        assert st == 0
        assert v == ref[k]


def test_select_invalid_k(engine):
    import torch
    ds = DeviceSort(np.arange(10, dtype=np.uint32), [], 0, 0, 32)
    torch.cuda.synchronize()
    assert engine.select_key(ds.data, 10)[0] == api.SortStatus.INVALID_VALUE
    assert engine.select_key(ds.data, -1)[0] == api.SortStatus.INVALID_VALUE

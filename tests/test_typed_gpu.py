"""sortArrayTyped: int32 and float32 keys sorted numerically through their
order-preserving uint32 image, keys returned as the caller's bit patterns,
value arrays and index mode moving with them (tolerance: exact)."""
import numpy as np
import pytest

from mgpu_old_b200 import api
from sortcase import DeviceSort

pytestmark = pytest.mark.gpu

SPECIAL_FLOATS = np.array([0x00000000, 0x80000000, 0x7f800000, 0xff800000, 0x7fc00000,
                           0xffc00000, 0x00000001, 0x80000001, 0x3f800000, 0xbf800000,
                           0x7f7fffff, 0xff7fffff], dtype=np.uint32)


def image(keys, kind):
    """The uint32 image, restated with numpy from its definition."""
    keys = keys.astype(np.uint32)
    if kind == api.KEY_INT32:
        return keys ^ np.uint32(0x80000000)
    neg = (keys >> np.uint32(31)) == 1
    return np.where(neg, ~keys, keys ^ np.uint32(0x80000000)).astype(np.uint32)


def float_keys(n, seed):
    rng = np.random.default_rng(seed)
    f = (rng.standard_normal(n) * 10.0 ** rng.integers(-30, 30, n)).astype(np.float32)
    k = f.view(np.uint32).copy()
    k[rng.integers(0, n, max(1, n // 50))] = SPECIAL_FLOATS[rng.integers(0, 12, max(1, n // 50))]
    k[::7] = k[0]   # duplicates
    return k


def int_keys(n, seed):
    rng = np.random.default_rng(seed)
    k = rng.integers(-2 ** 31, 2 ** 31, n, dtype=np.int64).astype(np.int32).view(np.uint32)
    ext = np.array([0x80000000, 0x7fffffff, 0, 0xffffffff, 1], dtype=np.uint32)
    k[rng.integers(0, n, max(1, n // 40))] = ext[rng.integers(0, 5, max(1, n // 40))]
    return k.copy()


def run_typed(engine, keys, values, vc, first, end, kind, early=False):
    import torch
    ds = DeviceSort(keys, values, vc, first, end, early_exit=early)
    torch.cuda.synchronize()
    st = engine.sort_array_typed(ds.data, kind)
    assert st == 0, api.sort_status_string(st)
    assert engine.synchronize() == 0
    torch.cuda.synchronize()
    return ds.result()


def expected(oracle_mod, keys, values, vc, first, end, kind):
    _, (perm,) = oracle_mod.sort_stable(image(keys, kind), [], -1, first, end)
    perm = perm.astype(np.int64)
    ek = keys[perm]
    if vc == -1:
        return ek, [perm.astype(np.uint32)]
    return ek, [v[perm] for v in values]


@pytest.mark.parametrize("kind", [api.KEY_FLOAT32, api.KEY_INT32])
@pytest.mark.parametrize("vc", [-1, 0, 1, 3])
@pytest.mark.parametrize("n", [1, 1000, 100_003])
def test_typed_matches_oracle(engine, oracle_mod, kind, vc, n):
    keys = float_keys(n, n + vc) if kind == api.KEY_FLOAT32 else int_keys(n, n + vc)
    rng = np.random.default_rng(n)
    values = [rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
              for _ in range(max(vc, 0))]
    k, v = run_typed(engine, keys, values, vc, 0, 32, kind)
    ek, ev = expected(oracle_mod, keys, values, vc, 0, 32, kind)
    assert np.array_equal(k, ek)
    for a, b in zip(v, ev):
        assert np.array_equal(a, b)


def test_float_order_is_numeric(engine, oracle_mod):
    n = 1 << 20
    keys = float_keys(n, 5)
    k, _ = run_typed(engine, keys, [], 0, 0, 32, api.KEY_FLOAT32)
    f = k.view(np.float32)
    ok = ~np.isnan(f)
    g = f[ok]
    assert (g[1:] >= g[:-1]).all()
    nan_pos = np.nonzero(~ok)[0]
    neg_nan = (k[nan_pos] >> 31) == 1
    # Negative NaNs first, positive NaNs last.
    assert (nan_pos[neg_nan] < np.nonzero(ok)[0].min()).all()
    assert (nan_pos[~neg_nan] > np.nonzero(ok)[0].max()).all()


def test_int_order_is_numeric(engine):
    keys = int_keys(300_000, 9)
    k, (idx,) = run_typed(engine, keys, [], -1, 0, 32, api.KEY_INT32)
    s = k.view(np.int32)
    assert np.array_equal(s, np.sort(keys.view(np.int32), kind="stable"))
    assert np.array_equal(idx, np.argsort(keys.view(np.int32), kind="stable").astype(np.uint32))


@pytest.mark.parametrize("first,end", [(16, 32), (0, 20), (31, 32)])
def test_typed_bit_range_of_image(engine, oracle_mod, first, end):
    keys = float_keys(50_000, first + end)
    k, (idx,) = run_typed(engine, keys, [], -1, first, end, api.KEY_FLOAT32)
    ek, (eidx,) = expected(oracle_mod, keys, [], -1, first, end, api.KEY_FLOAT32)
    assert np.array_equal(k, ek) and np.array_equal(idx, eidx)


def test_typed_early_exit_restores_keys(engine, oracle_mod):
    """Every pass skipped (one key repeated): the keys still come back as
    the caller's bit patterns."""
    keys = np.full(70_000, 0xbf800000, dtype=np.uint32)   # -1.0f
    k, (idx,) = run_typed(engine, keys, [], -1, 0, 32, api.KEY_FLOAT32, early=True)
    assert np.array_equal(k, keys)
    assert np.array_equal(idx, np.arange(keys.size, dtype=np.uint32))


def test_typed_invalid_key_type(engine):
    import torch
    keys = int_keys(1000, 1)
    ds = DeviceSort(keys, [], 0, 0, 32)
    torch.cuda.synchronize()
    assert engine.sort_array_typed(ds.data, 3) == api.SortStatus.INVALID_VALUE
    assert np.array_equal(ds.result()[0], keys)

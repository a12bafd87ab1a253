"""The alternative pass methods, bit for bit against the oracle's stable
sort: onesweep passes (MGPU_SORT_PASS=onesweep: one upsweep, then one
kernel per pass with a decoupled lookback) and the cooperative sort
(MGPU_SORT_COOP_MAX=<n>: every pass of a sort of at most n elements in one
launch with grid-wide barriers). Both are read when an engine is created, so
each test makes its own engine with the variable set; neither is the
default (the range partition measured faster on B200)."""
import os

import numpy as np
import pytest

from sortcase import run_sort

pytestmark = pytest.mark.gpu


def _engine_with(env):
    from mgpu_old_b200 import api
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return api.MgpuSort()
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _case(n, value_count, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    # Ties within the sorted field make stability visible.
    keys[rng.random(n) < 0.3] &= np.uint32(0xFFF0000F)
    arrays = max(value_count, 0)
    values = [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
              for _ in range(arrays)]
    return keys, values


def _check(engine, oracle_mod, n, value_count, first_bit, end_bit, seed):
    keys, values = _case(n, value_count, seed)
    ds = run_sort(engine, keys, values, value_count, first_bit, end_bit)
    got_k, got_v = ds.result()
    exp_k, exp_v = oracle_mod.sort_stable(keys, values, value_count, first_bit, end_bit)
    assert np.array_equal(got_k, exp_k)
    assert len(got_v) == len(exp_v)
    for a, b in zip(got_v, exp_v):
        assert np.array_equal(a, b)


ONESWEEP_CASES = [
    (5_000, 0, 0, 32, 1),
    (100_003, -1, 0, 32, 2),
    (1 << 20, 1, 3, 29, 3),
    (3_000_001, 1, 0, 32, 4),
    (250_007, 3, 0, 17, 5),
    (2_000_000, 0, 8, 24, 6),
]


@pytest.mark.parametrize("n,value_count,first_bit,end_bit,seed", ONESWEEP_CASES)
def test_onesweep_against_oracle(engine, oracle_mod, n, value_count, first_bit, end_bit,
                                 seed):
    e = _engine_with({"MGPU_SORT_PASS": "onesweep"})
    try:
        for _ in range(2):          # the second call replays a captured graph
            _check(e, oracle_mod, n, value_count, first_bit, end_bit, seed)
    finally:
        e.release()


COOP_CASES = [
    (4_097, 0, 0, 32, 11),
    (65_536, -1, 0, 32, 12),
    (1 << 20, 0, 0, 32, 13),
    (1_000_003, 1, 3, 29, 14),
    (3_999_999, 1, 0, 32, 15),
    (777_777, -1, 0, 17, 16),
]


@pytest.mark.parametrize("n,value_count,first_bit,end_bit,seed", COOP_CASES)
def test_cooperative_sort_against_oracle(engine, oracle_mod, n, value_count, first_bit,
                                         end_bit, seed):
    e = _engine_with({"MGPU_SORT_COOP_MAX": str(1 << 22)})
    try:
        for _ in range(2):
            _check(e, oracle_mod, n, value_count, first_bit, end_bit, seed)
    finally:
        e.release()

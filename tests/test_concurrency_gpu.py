"""Several engines sorting at once, each on its own stream: one-array sorts
above and below the small-array limit and segmented batches, with random
sizes, value modes and bit ranges, so that the engines' scratch buffers grow
and are freed while other engines' sorts run. Every result is checked bit
for bit against the oracle (one stable sort, or one per segment). Run with
the default pass method and with onesweep passes (MGPU_SORT_PASS=onesweep,
which adds the lookback buffers to the scratch that grows)."""
import os

import numpy as np
import pytest

from sortcase import DeviceSort

pytestmark = pytest.mark.gpu

ENGINES = 4
ROUNDS = 40


def _make_engines(env):
    from mgpu_old_b200 import api
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return [api.MgpuSort() for _ in range(ENGINES)]
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def _job(rng):
    import torch
    kind = int(rng.integers(0, 3))          # 0 one array, 1 small array, 2 segmented
    n = int(rng.integers(1, 4097)) if kind == 1 else int(rng.integers(4097, 300_000))
    value_count = int(rng.choice([-1, 0, 1, 2]))
    end_bit = int(rng.choice([16, 24, 32]))
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    keys[::4] &= np.uint32(0x00FFFF00)      # ties in the sorted field
    arrays = max(value_count, 0)
    values = [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
              for _ in range(arrays)]
    ds = DeviceSort(keys, values, value_count, 0, end_bit, cap=n)
    offsets = None
    if kind == 2:
        cuts = np.sort(rng.integers(0, n, int(rng.integers(2, 60))))
        offsets = np.concatenate([[0], cuts, [n]]).astype(np.int32)
        ds.offsets_dev = torch.from_numpy(offsets).cuda()
    return ds, keys, values, value_count, end_bit, offsets


@pytest.mark.parametrize("method", ["range", "onesweep"])
def test_engines_on_their_own_streams(engine, oracle_mod, method):
    import torch
    from mgpu_old_b200 import api
    env = {"MGPU_SORT_PASS": method}
    engines = _make_engines(env)
    streams = [torch.cuda.Stream() for _ in engines]
    rng = np.random.Generator(np.random.MT19937(2024 if method == "range" else 2025))
    try:
        for _ in range(ROUNDS):
            jobs = [_job(rng) for _ in engines]
            torch.cuda.synchronize()
            for e, s, (ds, _, _, _, _, offsets) in zip(engines, streams, jobs):
                if offsets is None:
                    st = e.sort_array_async(ds.data, s.cuda_stream)
                else:
                    st = e.sort_segmented(ds.data, ds.offsets_dev.data_ptr(),
                                          offsets.size - 1, s.cuda_stream)
                assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
            for e in engines:
                st = e.synchronize()
                assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
            torch.cuda.synchronize()
            for ds, keys, values, value_count, end_bit, offsets in jobs:
                got_k, got_v = ds.result()
                if offsets is None:
                    exp_k, exp_v = oracle_mod.sort_stable(keys, values, value_count, 0,
                                                          end_bit)
                else:
                    exp_k, exp_v = oracle_mod.sort_segments(keys, values, value_count,
                                                            offsets, 0, end_bit)
                assert np.array_equal(got_k, exp_k)
                for a, b in zip(got_v, exp_v):
                    assert np.array_equal(a, b)
    finally:
        for e in engines:
            e.release()

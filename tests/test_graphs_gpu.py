"""Repeated sorts replay a captured CUDA graph of their launch sequence
(sortEnableGraphs, sortGraphStats): results stay equal to the oracle's with
new buffer contents, new segment boundaries behind the same offsets
pointer, changed shapes in between, and with graphs turned off
(tolerance: exact)."""
import numpy as np
import pytest

from mgpu_old_b200 import api
from sortcase import DeviceSort

pytestmark = pytest.mark.gpu


@pytest.fixture()
def fresh_engine(engine):
    e = api.MgpuSort()
    yield e
    e.release()


def load_inputs(ds, keys, values):
    import torch
    t, off = ds.tensors[ds.data.keys[0]]
    t[off:off + keys.size] = torch.from_numpy(keys.view(np.int32)).cuda()
    for i, v in enumerate(values):
        t, off = ds.tensors[ds.data.values[i][0]]
        t[off:off + v.size] = torch.from_numpy(v.view(np.int32)).cuda()


def test_repeated_sort_replays_graph(fresh_engine, oracle_mod):
    import torch
    n = 300_000
    ds = DeviceSort(np.zeros(n, np.uint32), [np.zeros(n, np.uint32)], 1, 0, 32)
    rng = np.random.default_rng(1)
    for it in range(6):
        # Parity returns to the start after an even pass count (4 passes),
        # so every call has the same launch sequence.
        keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        vals = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        load_inputs(ds, keys, [vals])
        torch.cuda.synchronize()
        assert fresh_engine.sort_array(ds.data) == 0
        assert fresh_engine.synchronize() == 0
        torch.cuda.synchronize()
        k, (v,) = ds.result()
        ek, (ev,) = oracle_mod.sort_stable(keys, [vals], 1, 0, 32)
        assert np.array_equal(k, ek) and np.array_equal(v, ev)
    replays, cached = fresh_engine.graph_stats()
    assert cached >= 1
    assert replays >= 4


def test_odd_pass_count_alternates_two_graphs(fresh_engine, oracle_mod):
    """Three passes swap the buffers: calls alternate between two launch
    sequences, each captured once."""
    import torch
    n = 100_000
    ds = DeviceSort(np.zeros(n, np.uint32), [], -1, 0, 24)
    rng = np.random.default_rng(2)
    for it in range(8):
        keys = rng.integers(0, 2 ** 24, n, dtype=np.uint64).astype(np.uint32)
        # The result of the previous call sits in keys[0]; load over it.
        load_inputs(ds, keys, [])
        torch.cuda.synchronize()
        assert fresh_engine.sort_array(ds.data) == 0
        assert fresh_engine.synchronize() == 0
        torch.cuda.synchronize()
        k, (idx,) = ds.result()
        ek, (eidx,) = oracle_mod.sort_stable(keys, [], -1, 0, 24)
        assert np.array_equal(k, ek) and np.array_equal(idx, eidx)
    replays, cached = fresh_engine.graph_stats()
    assert cached == 2
    assert replays >= 4


def test_segmented_replay_with_new_boundaries(fresh_engine, oracle_mod):
    import torch
    n, segs = 200_000, 300
    ds = DeviceSort(np.zeros(n, np.uint32), [np.zeros(n, np.uint32)], 1, 0, 32)
    offs_t = torch.zeros(segs + 1, dtype=torch.int32, device="cuda")
    rng = np.random.default_rng(3)
    for it in range(6):
        cuts = np.sort(rng.choice(np.arange(1, n), segs - 1, replace=False))
        offs = np.concatenate([[0], cuts, [n]]).astype(np.int32)
        offs_t.copy_(torch.from_numpy(offs))
        keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        vals = np.arange(n, dtype=np.uint32)
        load_inputs(ds, keys, [vals])
        torch.cuda.synchronize()
        assert fresh_engine.sort_segmented(ds.data, offs_t.data_ptr(), segs) == 0
        assert fresh_engine.synchronize() == 0
        torch.cuda.synchronize()
        k, (v,) = ds.result()
        ek, (ev,) = oracle_mod.sort_segments(keys, [vals], 1, offs, 0, 32)
        assert np.array_equal(k, ek) and np.array_equal(v, ev)
    assert fresh_engine.graph_stats()[0] >= 4


def test_graphs_off_and_shape_changes(fresh_engine, oracle_mod):
    import torch
    rng = np.random.default_rng(4)
    for enable in (True, False, True):
        assert fresh_engine.enable_graphs(enable) == 0
        for n in (5000, 77_777, 5000, 77_777, 5000):
            keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
            ds = DeviceSort(keys, [], 0, 3, 29)
            torch.cuda.synchronize()
            assert fresh_engine.sort_array(ds.data) == 0
            assert fresh_engine.synchronize() == 0
            torch.cuda.synchronize()
            ek, _ = oracle_mod.sort_stable(keys, [], 0, 3, 29)
            assert np.array_equal(ds.result()[0], ek)
        if not enable:
            assert fresh_engine.graph_stats()[1] == 0


def test_typed_sort_replays_graph(fresh_engine, oracle_mod):
    """sortArrayTyped (float keys) repeated on the same buffers: the key
    transforms are part of the captured sequence."""
    import torch
    n = 70_000
    ds = DeviceSort(np.zeros(n, np.uint32), [np.zeros(n, np.uint32)], 1, 0, 32)
    rng = np.random.default_rng(5)
    for it in range(5):
        f = (rng.standard_normal(n) * 1e3).astype(np.float32)
        keys = f.view(np.uint32).copy()
        vals = np.arange(n, dtype=np.uint32)
        load_inputs(ds, keys, [vals])
        torch.cuda.synchronize()
        assert fresh_engine.sort_array_typed(ds.data, api.KEY_FLOAT32) == 0
        assert fresh_engine.synchronize() == 0
        torch.cuda.synchronize()
        k, (v,) = ds.result()
        order = np.argsort(f, kind="stable")
        assert np.array_equal(v, order.astype(np.uint32))
        assert np.array_equal(k, keys[order])
    assert fresh_engine.graph_stats()[0] >= 3

"""Helpers for the GPU tests: put a sort case into device buffers (torch
allocations), run it through the C ABI and read the result back."""
from __future__ import annotations

import numpy as np

from mgpu_old_b200 import api

ROUND = 2048


def round_up(x: int, m: int = ROUND) -> int:
    return (x + m - 1) // m * m


def to_dev(a: np.ndarray, cap: int, offset: int = 0):
    """uint32 host array -> int32 cuda tensor of cap + offset elements whose
    [offset, offset + len) holds a; returns (tensor, device pointer)."""
    import torch
    t = torch.full((cap + offset,), -1, dtype=torch.int32, device="cuda")
    if a.size:
        t[offset:offset + a.size] = torch.from_numpy(a.view(np.int32)).cuda()
    return t, t.data_ptr() + 4 * offset


class DeviceSort:
    """A sortData_d whose buffers are torch allocations owned by this object."""

    def __init__(self, keys, values, value_count, first_bit, end_bit,
                 offset: int = 0, early_exit: bool = False, cap: int | None = None):
        n = int(keys.size)
        self.n = n
        cap = cap if cap is not None else round_up(max(n, 1))
        self.tensors = {}
        d = api.SortData()
        d.maxElements = cap
        d.numElements = n
        d.valueCount = value_count
        d.firstBit = first_bit
        d.endBit = end_bit
        d.earlyExit = early_exit
        d.parity = 0
        arrays = 1 if value_count == -1 else max(value_count, 0)
        k0, p0 = to_dev(np.asarray(keys, np.uint32), cap, offset)
        k1, p1 = to_dev(np.zeros(0, np.uint32), cap, offset)
        d.keys[0], d.keys[1] = p0, p1
        self.tensors[p0] = (k0, offset)
        self.tensors[p1] = (k1, offset)
        for i in range(arrays):
            src = values[i] if value_count != -1 else np.zeros(0, np.uint32)
            v0, q0 = to_dev(np.asarray(src, np.uint32), cap, offset)
            v1, q1 = to_dev(np.zeros(0, np.uint32), cap, offset)
            d.values[i][0], d.values[i][1] = q0, q1
            self.tensors[q0] = (v0, offset)
            self.tensors[q1] = (v1, offset)
        self.data = d
        self.arrays = arrays
        self.original_keys_ptr = p0

    def read(self, ptr: int, count: int | None = None) -> np.ndarray:
        t, off = self.tensors[ptr]
        count = self.n if count is None else count
        return t[off:off + count].cpu().numpy().view(np.uint32).copy()

    def read_full(self, ptr: int) -> np.ndarray:
        t, off = self.tensors[ptr]
        return t.cpu().numpy().view(np.uint32).copy()

    def result(self):
        keys = self.read(self.data.keys[0])
        vals = [self.read(self.data.values[i][0]) for i in range(self.arrays)]
        return keys, vals


def run_sort(engine, keys, values, value_count, first_bit, end_bit, how="array",
             bit_pass=6, num_threads=256, early_exit=False, offset=0):
    import torch
    ds = DeviceSort(keys, values, value_count, first_bit, end_bit, offset=offset,
                    early_exit=early_exit)
    torch.cuda.synchronize()
    if how == "array":
        st = engine.sort_array(ds.data)
    elif how == "ex":
        st = engine.sort_array_ex(ds.data, num_threads, 8, bit_pass)
    else:
        raise ValueError(how)
    assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
    st = engine.synchronize()
    assert st == api.SortStatus.SUCCESS, api.sort_status_string(st)
    torch.cuda.synchronize()
    return ds


def check_index_result(keys_in, first_bit, end_bit, keys_out, idx_out):
    """Size-independent proof that (keys_out, idx_out) is THE stable sort of
    keys_in by the bit field: idx_out is a permutation, keys_out gathers
    through it, fields are non-decreasing, equal fields keep index order."""
    n = keys_in.size
    assert idx_out.size == n
    assert np.array_equal(np.sort(idx_out), np.arange(n, dtype=np.uint32))
    assert np.array_equal(keys_out, keys_in[idx_out])
    bits = end_bit - first_bit
    mask = np.uint32(0xFFFFFFFF if bits >= 32 else (1 << bits) - 1)
    f = (keys_out >> np.uint32(first_bit)) & mask
    if n > 1:
        df = f[1:].astype(np.int64) - f[:-1].astype(np.int64)
        assert (df >= 0).all()
        eq = df == 0
        assert (idx_out[1:][eq] > idx_out[:-1][eq]).all()

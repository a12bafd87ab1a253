"""The BWT block sort (include/mgpubwt.h) through the C ABI: rotation order,
transform and tie-group statistics against the oracle, over the host-only
and GPU paths, every key-stream count and block kinds with many ties
(tolerance: exact; avSegSize to float rounding)."""
import ctypes

import numpy as np
import pytest

from mgpu_old_b200.workloads import text_block

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bwt(engine):
    from mgpu_old_b200 import api
    e = api.BwtEngine()
    yield e
    e.close()


def block_of(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "bytes":
        return rng.integers(0, 256, n).astype(np.uint8)
    if kind == "dna":
        return np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, n)].copy()
    if kind == "text":
        return text_block(n, seed)
    if kind == "periodic":
        return np.frombuffer((b"mississippi" * (n // 11 + 1))[:n], dtype=np.uint8).copy()
    if kind == "runs":
        return np.repeat(rng.integers(0, 3, n // 50 + 1).astype(np.uint8), 50)[:n].copy()
    raise ValueError(kind)


def check(bwt, oracle_mod, blk, key_size):
    st, idx, xf, seg, av = bwt.sort_block(blk, key_size)
    assert st == 0
    e_idx, e_xf, e_seg, e_av = oracle_mod.bwt(blk, key_size)
    assert np.array_equal(xf, e_xf)
    assert np.array_equal(idx, e_idx)
    assert seg == e_seg
    assert av == pytest.approx(e_av, rel=1e-6)


@pytest.mark.parametrize("key_size", [1, 3, 4, 5, 8, 12, 13, 16, 24])
@pytest.mark.parametrize("kind", ["bytes", "dna", "text"])
def test_bwt_matches_oracle(bwt, oracle_mod, kind, key_size):
    check(bwt, oracle_mod, block_of(kind, 60_000, key_size), key_size)


@pytest.mark.parametrize("n", [0, 1, 2, 100, 2999, 3000, 3001, 7681, 250_000])
def test_bwt_sizes(bwt, oracle_mod, n):
    """Host-only blocks below 3000 bytes, GPU blocks from 3000 (partial
    tiles, a block larger than one pass range)."""
    check(bwt, oracle_mod, block_of("text", n, n), 8)


@pytest.mark.parametrize("kind", ["periodic", "runs"])
def test_bwt_ties(bwt, oracle_mod, kind):
    """Blocks whose rotations tie on long prefixes or as whole strings."""
    check(bwt, oracle_mod, block_of(kind, 20_000, 3), 6)


def test_bwt_transform_may_alias_block(bwt, oracle_mod, lib):
    blk = block_of("dna", 9000, 11)
    _, e_xf, _, _ = oracle_mod.bwt(blk, 4)
    buf = blk.copy()
    st = lib.bwtSortBlock(bwt._engine, buf.ctypes.data_as(ctypes.c_void_p), buf.size, 4,
                          buf.ctypes.data_as(ctypes.c_void_p), None, None, None)
    assert st == 0
    assert np.array_equal(buf, e_xf)


def test_bwt_invalid_arguments(bwt):
    from mgpu_old_b200 import api
    big = block_of("bytes", 5000, 1)
    for ks in (0, 25):
        assert bwt.sort_block(big, ks)[0] == api.BwtStatus.INVALID_VALUE
    # Below 3000 bytes the block never reaches the key-size check
    # (mgpubwt.cpp:217-225).
    assert bwt.sort_block(big[:100], 25)[0] == api.BwtStatus.SUCCESS


def test_bwt_repeated_blocks(bwt, oracle_mod):
    """One engine, blocks of different sizes and key sizes in a row."""
    for n, ks in [(50_000, 16), (4000, 2), (120_000, 24), (3000, 9)]:
        check(bwt, oracle_mod, block_of("text", n, n + ks), ks)

"""CPU checks of the oracle: committed golden fixtures, the reference's own
cpusort.cpp (when built here), and agreement of its two restatements."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_fixture(path):
    z = np.load(path)
    vc = int(z["value_count"])
    arrays = 1 if vc == -1 else vc
    vals = [z[f"values{i}"] for i in range(vc)] if vc > 0 else []
    exp_vals = [z[f"expect_values{i}"] for i in range(arrays)]
    return (z["keys"], vals, vc, int(z["first_bit"]), int(z["end_bit"]),
            z["expect_keys"], exp_vals)


def split_bits(bits):
    if bits <= 0:
        return []
    p = (bits + 7) // 8
    return [bits // p + (i < bits % p) for i in range(p)]


def test_fixtures_present():
    assert len(FIXTURES) >= 10


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f) for f in FIXTURES])
def test_oracle_matches_golden(oracle_mod, path):
    keys, vals, vc, fb, eb, ek, ev = load_fixture(path)
    k, v = oracle_mod.sort_stable(keys, vals, vc, fb, eb)
    assert np.array_equal(k, ek)
    for a, b in zip(v, ev):
        assert np.array_equal(a, b)
    k2, v2 = oracle_mod.sort_lsd(keys, vals, vc, fb, split_bits(eb - fb), 512, 3)
    assert np.array_equal(k2, ek)
    for a, b in zip(v2, ev):
        assert np.array_equal(a, b)


def _ref_or_skip(oracle_mod):
    r = oracle_mod.ref_lib()
    if r is None:
        pytest.skip("reference cpusort.cpp not built here")
    return r


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 1000, 20000])
def test_oracle_matches_reference_sort2(oracle_mod, n):
    r = _ref_or_skip(oracle_mod)
    rng = np.random.Generator(np.random.MT19937(n))
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    ref = keys.copy()
    r.ref_cpusort_sort2(oracle_mod._p(ref), n, 64)
    k, _ = oracle_mod.sort_stable(keys, [], 0, 0, 32)
    assert np.array_equal(k, ref)
    assert np.array_equal(oracle_mod.std_sort_keys(keys), ref)


@pytest.mark.parametrize("first,end", [(0, 8), (3, 17), (7, 25), (13, 32), (31, 32), (0, 32)])
def test_oracle_matches_reference_bit_ranges(oracle_mod, first, end):
    """Chained reference Sort2Pass calls over [first, end) sort keys stably by
    that field (keys outside the field make ties visible)."""
    r = _ref_or_skip(oracle_mod)
    rng = np.random.Generator(np.random.MT19937(first * 100 + end))
    keys = rng.integers(0, 1 << 32, 7777, dtype=np.uint64).astype(np.uint32)
    keys[::3] &= np.uint32(0xF0F0F0F0)   # more ties
    ref = keys.copy()
    bit = first
    for w in split_bits(end - first):
        r.ref_cpusort_sort2pass(oracle_mod._p(ref), bit, w, ref.size, 256)
        bit += w
    k, _ = oracle_mod.sort_stable(keys, [], 0, first, end)
    assert np.array_equal(k, ref)


@pytest.mark.parametrize("vc", [-1, 0, 1, 2, 6])
@pytest.mark.parametrize("first,end", [(0, 32), (5, 23), (24, 32)])
def test_oracle_restatements_agree(oracle_mod, vc, first, end):
    rng = np.random.Generator(np.random.MT19937(vc + 10 * first + end))
    n = 9000
    keys = rng.integers(0, 1 << 20, n, dtype=np.uint64).astype(np.uint32) << np.uint32(9)
    vals = [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
            for _ in range(max(vc, 0))]
    k1, v1 = oracle_mod.sort_stable(keys, vals, vc, first, end)
    for widths in (split_bits(end - first), [1] * (end - first)):
        k2, v2 = oracle_mod.sort_lsd(keys, vals, vc, first, widths, 1000, 4)
        assert np.array_equal(k1, k2)
        for a, b in zip(v1, v2):
            assert np.array_equal(a, b)


def test_oracle_catches_a_planted_mistake(oracle_mod):
    """The checker must notice an unstable result: swap two tied elements."""
    keys = np.array([5, 1, 5, 1], np.uint32)
    idx = np.arange(4, dtype=np.uint32)
    k, (v,) = oracle_mod.sort_stable(keys, [idx], 1, 0, 32)
    assert list(v) == [1, 3, 0, 2]
    bad = v.copy()
    bad[[0, 1]] = bad[[1, 0]]
    assert not np.array_equal(bad, v)


def test_oracle_index_mode_empty_range(oracle_mod):
    keys = np.array([3, 1, 2], np.uint32)
    k, (v,) = oracle_mod.sort_stable(keys, [], -1, 4, 4)
    assert list(k) == [3, 1, 2] and list(v) == [0, 1, 2]


# Burrows-Wheeler block sort (the BWT caller of sortArray).

from mgpu_old_b200.workloads import text_block  # noqa: E402

def test_oracle_bwt_known_answers(oracle_mod):
    # Cyclic BWT of two classic strings.
    idx, xf, seg, av = oracle_mod.bwt(b"banana", 4)
    assert list(idx) == [5, 3, 1, 0, 4, 2]
    assert bytes(xf) == b"nnbaaa"
    assert (seg, av) == (1, 6.0)
    idx, xf, _, _ = oracle_mod.bwt(b"abracadabra", 1)
    assert bytes(xf) == b"rdarcaaaabb"


@pytest.mark.parametrize("kind", ["random4", "text", "periodic"])
@pytest.mark.parametrize("n", [2, 17, 4000])
def test_oracle_bwt_matches_reference_quicksort(oracle_mod, kind, n):
    """Against the reference BWT library's own string quicksort
    (bwt/src/mgpubwt/cpusort.cpp) over all rotations, built here."""
    if oracle_mod.ref_bwt_lib() is None:
        pytest.skip("reference BWT cpusort.cpp not built here")
    rng = np.random.default_rng(n)
    if kind == "random4":
        blk = rng.integers(0, 4, n).astype(np.uint8)
    elif kind == "text":
        blk = text_block(n, n)
    else:
        blk = np.frombuffer((b"abcab" * (n // 5 + 1))[:n], dtype=np.uint8).copy()
    idx, xf, _, _ = oracle_mod.bwt(blk, 8)
    ref_idx, ref_xf = oracle_mod.ref_bwt_block(blk)
    assert np.array_equal(xf, ref_xf)
    # Rotations equal as whole strings may be ordered differently by the
    # quicksort; every other position must agree.
    sym = np.concatenate([blk, blk])
    for i in np.nonzero(idx != ref_idx)[0]:
        assert bytes(sym[idx[i]:idx[i] + n]) == bytes(sym[ref_idx[i]:ref_idx[i] + n])


def test_key_image_round_trip_and_order():
    """The host restatement of the int32/float32 key image (used by the
    bench's checks): a bijection that orders numerically."""
    from mgpu_old_b200 import workloads as w
    rng = np.random.default_rng(1)
    k = rng.integers(0, 2 ** 32, 100_000, dtype=np.uint64).astype(np.uint32)
    for t in (0, 1, 2):
        assert np.array_equal(w.key_preimage(w.key_image(k, t), t), k)
    f = np.array([-np.inf, -1.5, -1e-40, -0.0, 0.0, 1e-40, 2.0, np.inf],
                 dtype=np.float32).view(np.uint32)
    assert (np.diff(w.key_image(f, 2).astype(np.int64)) > 0).all()
    i = np.array([-2 ** 31, -1, 0, 1, 2 ** 31 - 1], dtype=np.int32).view(np.uint32)
    assert (np.diff(w.key_image(i, 1).astype(np.int64)) > 0).all()


def test_workload_generators_fields():
    """Workload dataclasses keep their fields in place (segment offsets,
    key types) at small sizes."""
    from mgpu_old_b200 import workloads as w
    seg = w.segments_lognormal(50)
    assert seg.offsets is not None and seg.offsets.size == 51 and seg.key_type == 0
    assert int(seg.offsets[-1]) == seg.n
    f = w.pairs_float32(1000)
    assert f.key_type == 2 and f.value_count == 1
    assert w.pairs_and24(1000).key_type == 0

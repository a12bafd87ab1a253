"""Seeded synthetic inputs for the sort workloads (numpy, host memory).

Each generator returns host arrays of the workload's shape and value
distribution. There is no public dataset for this path; these stand in for
the reference's own benchmark inputs (uniform random keys, value = index,
sort/src/testsort/testsort.cpp:176-194).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class SortCase:
    name: str
    keys: np.ndarray
    values: list[np.ndarray] = field(default_factory=list)
    value_count: int = 0          # -1 index mode, 0 keys only, 1..6
    first_bit: int = 0
    end_bit: int = 32
    key_type: int = 0             # 0 uint32, 1 int32, 2 float32 (sortArrayTyped)

    @property
    def n(self) -> int:
        return int(self.keys.size)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.MT19937(seed))


def _u32(rng: np.random.Generator, n: int, high: int = 1 << 32) -> np.ndarray:
    return rng.integers(0, high, size=n, dtype=np.uint64).astype(np.uint32)


def keys_uniform32(n: int = 1 << 20, seed: int = 1) -> SortCase:
    """Keys-only, uniform over 32 bits, [0, 32). 1,048,576 keys by default."""
    return SortCase("keys_u32_1M" if n == 1 << 20 else f"keys_u32_{n}",
                    _u32(_rng(seed), n))


def pairs_and24(n: int = 1 << 25, seed: int = 2) -> SortCase:
    """Key-value: key = (r1 & r2) & 0xFFFFFF (skewed digits), value = index,
    bits [0, 24). 33,554,432 pairs by default."""
    rng = _rng(seed)
    keys = (_u32(rng, n) & _u32(rng, n)) & np.uint32(0x00FFFFFF)
    return SortCase("pairs_and24_32M" if n == 1 << 25 else f"pairs_and24_{n}",
                    keys, [np.arange(n, dtype=np.uint32)], 1, 0, 24)


def multi6_17bit(n: int = 1 << 24, seed: int = 3) -> SortCase:
    """Key + 6 value arrays: keys uniform in [0, 2^17) (heavy duplicates),
    random payloads, full 32-bit range. 16,777,216 keys by default."""
    rng = _rng(seed)
    keys = _u32(rng, n, 1 << 17)
    vals = [_u32(rng, n) for _ in range(6)]
    return SortCase("multi6_17bit_16M" if n == 1 << 24 else f"multi6_17bit_{n}",
                    keys, vals, 6, 0, 32)


def pairs_uniform32(n: int = 1 << 26, seed: int = 5) -> SortCase:
    """Key-value, uniform 32-bit keys, value = index, [0, 32). 64M pairs."""
    rng = _rng(seed)
    return SortCase("pairs_u32_64M" if n == 1 << 26 else f"pairs_u32_{n}",
                    _u32(rng, n), [np.arange(n, dtype=np.uint32)], 1, 0, 32)


def lognormal_segment_sizes(num_segments: int = 10_000, median: float = 2048.0,
                            sigma: float = 2.0, lo: int = 1, hi: int = 4_194_304,
                            seed: int = 4) -> np.ndarray:
    """Segment sizes round(lognormal(ln median, sigma)) clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = np.rint(rng.lognormal(np.log(median), sigma, num_segments))
    return np.clip(sizes, lo, hi).astype(np.int64)


@dataclass
class SegmentedCase(SortCase):
    offsets: np.ndarray = None   # int32, num_segments + 1 boundaries

    @property
    def num_segments(self) -> int:
        return int(self.offsets.size - 1)


def segments_lognormal(num_segments: int = 10_000, seed: int = 4,
                       scale_to: int | None = None) -> SegmentedCase:
    """Batched segmented sort: lognormal segment sizes (median 2048, sigma 2,
    clipped to [1, 4194304]), uniform 32-bit keys, value = index within the
    segment, bits [0, 32). scale_to rescales the sizes to that total."""
    sizes = lognormal_segment_sizes(num_segments, seed=seed)
    if scale_to:
        sizes = np.maximum(1, np.rint(sizes * (scale_to / sizes.sum()))).astype(np.int64)
    offsets = np.zeros(sizes.size + 1, np.int64)
    np.cumsum(sizes, out=offsets[1:])
    n = int(offsets[-1])
    keys = _u32(_rng(seed + 100), n)
    local = (np.arange(n, dtype=np.int64) - np.repeat(offsets[:-1], sizes)).astype(np.uint32)
    name = f"segments_{num_segments}_lognormal" + (f"_scaled{scale_to}" if scale_to else "")
    return SegmentedCase(name, keys, [local], 1, 0, 32, offsets=offsets.astype(np.int32))


def key_image(keys: np.ndarray, key_type: int) -> np.ndarray:
    """The order-preserving uint32 image of int32 (1) or float32 (2) key
    bit patterns (identity for uint32)."""
    keys = np.asarray(keys, dtype=np.uint32)
    if key_type == 1:
        return keys ^ np.uint32(0x80000000)
    if key_type == 2:
        neg = (keys >> np.uint32(31)) == 1
        return np.where(neg, ~keys, keys ^ np.uint32(0x80000000)).astype(np.uint32)
    return keys


def key_preimage(image: np.ndarray, key_type: int) -> np.ndarray:
    """Inverse of key_image."""
    image = np.asarray(image, dtype=np.uint32)
    if key_type == 1:
        return image ^ np.uint32(0x80000000)
    if key_type == 2:
        pos = (image >> np.uint32(31)) == 1
        return np.where(pos, image ^ np.uint32(0x80000000), ~image).astype(np.uint32)
    return image


def pairs_float32(n: int = 1 << 25, seed: int = 10) -> SortCase:
    """Key-value with float32 keys (sortArrayTyped): normal values scaled by
    10^[-30, 30), value = index, full 32-bit image. 33,554,432 pairs."""
    rng = np.random.default_rng(seed)
    f = (rng.standard_normal(n) * 10.0 ** rng.integers(-30, 30, n)).astype(np.float32)
    return SortCase("pairs_f32_32M" if n == 1 << 25 else f"pairs_f32_{n}",
                    f.view(np.uint32).copy(), [np.arange(n, dtype=np.uint32)], 1, 0, 32,
                    key_type=2)


def keys_uniform32_64m() -> SortCase:
    """Keys-only, uniform over 32 bits, 64Mi keys (a large keys-only case)."""
    c = keys_uniform32(1 << 26, seed=6)
    c.name = "keys_u32_64M"
    return c


def text_block(n: int, seed: int = 7) -> np.ndarray:
    """Seeded English-like bytes for the BWT block sort: words from a
    generated 500-word vocabulary (1-8 letters, letter order by English
    frequency) drawn with Zipf(1.3) frequencies, separated by spaces and, one
    time in 12, newlines. Stands in for the reference's text test block."""
    rng = np.random.default_rng(seed)
    letters = np.frombuffer(b"etaoinshrdlcumwfgypbvkjxqz", dtype=np.uint8)
    vocab = [bytes(letters[rng.integers(0, 26, int(rng.integers(1, 9)))].tolist())
             for _ in range(500)]
    picks = np.minimum(rng.zipf(1.3, size=n // 2 + 16), 500) - 1
    seps = rng.random(picks.size) < 1 / 12
    out = bytearray()
    for w, nl in zip(picks, seps):
        out += vocab[int(w)]
        out += b"\n" if nl else b" "
        if len(out) >= n:
            break
    while len(out) < n:
        out += out[:n - len(out)]
    return np.frombuffer(bytes(out[:n]), dtype=np.uint8).copy()


WORKLOADS = {
    "keys_u32_1M": keys_uniform32,
    "pairs_and24_32M": pairs_and24,
    "multi6_17bit_16M": multi6_17bit,
    "pairs_u32_64M": pairs_uniform32,
    "keys_u32_64M": keys_uniform32_64m,
    "pairs_f32_32M": pairs_float32,
    "segments_10k": segments_lognormal,
    "segments_10k_64M": lambda: segments_lognormal(scale_to=1 << 26),
}


def algorithmic_bytes(n: int, first_bit: int, end_bit: int, value_count: int) -> int:
    """Canonical bytes of a sort: one key read for the histograms plus, per
    8-bit pass, one read and one write of every key and value:
    N * (4 + 2 * P * (4 + 4V)), P = ceil(bits / 8), index mode V = 1."""
    p = (end_bit - first_bit + 7) // 8
    v = 1 if value_count == -1 else value_count
    return n * (4 + 2 * p * (4 + 4 * v))

"""The segmented sort sizes its range table for seg_max_ranges(n, S) =
n / kMinTile + S + 1 ranges (sort_kernels.cu), and its plan kernel cuts
every segment of more than 4096 elements into min(64, ceil(tiles / 4))
ranges of tiles on the 16-byte grid from the segment's aligned-down start.
This restates that arithmetic on the CPU and checks the bound over random
and adversarial segmentations, for the tile sizes tile_config.h builds."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CONFIG = os.path.join(ROOT, "mgpu_old_b200", "csrc", "tile_config.h")

SMALL_MAX = 4096
MAX_RANGES_PER_SEGMENT = 64
TILES_PER_RANGE = 4


def _define(name):
    text = open(CONFIG).read()
    m = re.search(rf"#ifndef {name}\n#define {name} (\d+)", text)
    assert m, name
    return int(m.group(1))


def _tiles():
    """Tiles of the segmented passes' classes: keys only, the segmented
    single class (index mode, one value array), several value arrays."""
    keys = _define("MGPU_SORT_KEYS_THREADS") * _define("MGPU_SORT_KEYS_ITEMS")
    seg = _define("MGPU_SORT_SEG_SINGLE_THREADS") * _define("MGPU_SORT_SEG_SINGLE_ITEMS")
    multi = _define("MGPU_SORT_MULTI_THREADS") * _define("MGPU_SORT_MULTI_ITEMS")
    return [keys, seg, multi]


def _plan_ranges(offsets, tile):
    total = 0
    for b, e in zip(offsets[:-1], offsets[1:]):
        length = e - b
        if length <= SMALL_MAX:
            continue
        base = b & ~3
        tiles = (e - base + tile - 1) // tile
        total += min(MAX_RANGES_PER_SEGMENT, (tiles + TILES_PER_RANGE - 1) // TILES_PER_RANGE)
    return total


def _bound(n, segments, min_tile):
    return n // min_tile + segments + 1


def _segmentations(rng):
    # Lognormal sizes as the benchmark's batch.
    sizes = np.clip(np.round(rng.lognormal(np.log(2048), 2.0, 10_000)), 1, 1 << 22)
    yield sizes.astype(np.int64)
    # Just over the small-segment limit, shifted off the 16-byte grid.
    yield np.array([3] + [SMALL_MAX + 1] * 5000, dtype=np.int64)
    # One tile plus one element, many times: the most partial tiles.
    for t in _tiles():
        yield np.array([1] + [t + 1] * 2000, dtype=np.int64)
        yield np.array([2] + [4 * t + 1] * 500, dtype=np.int64)
        # Long enough for the 64-range cap.
        yield np.array([64 * 4 * t + 3] * 20, dtype=np.int64)
    # Random mixtures.
    for _ in range(20):
        yield rng.integers(1, 200_000, int(rng.integers(2, 3000)), dtype=np.int64)


def test_min_tile_condition():
    # The bound's proof needs the smallest tile to be at most 3 x 4096.
    assert min(_tiles()) <= 12288


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_plan_ranges_fit_the_scratch(seed):
    rng = np.random.default_rng(seed)
    tiles = _tiles()
    min_tile = min(tiles)
    for sizes in _segmentations(rng):
        offsets = np.concatenate([[0], np.cumsum(sizes)]).tolist()
        n, segments = offsets[-1], len(sizes)
        for tile in tiles:
            assert _plan_ranges(offsets, tile) <= _bound(n, segments, min_tile), (tile, n)

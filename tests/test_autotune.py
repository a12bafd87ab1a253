"""CPU checks of the autotuner's selection and header rewrite
(mgpu_old_b200/autotune.py); the measurement itself needs a B200."""
import json
import os
import shutil

from mgpu_old_b200 import autotune


def test_choose_takes_the_best_geometric_mean():
    table = {"a": {"x": 1.0, "y": 2.0}, "b": {"x": 1.1, "y": 1.5}, "c": {"x": 3.0}}
    winner, scores = autotune.choose(table)
    assert winner == "b"
    assert "c" not in scores          # a candidate missing a workload is not scored
    assert abs(scores["a"] - (1.0 * 2.0 / 1.5) ** 0.5) < 1e-12


def test_write_rewrites_only_the_winners(tmp_path):
    header = tmp_path / "tile_config.h"
    shutil.copy(autotune.CONFIG_H, header)
    results = {"multi": {"768x8x1": {"w": 2.0}, "512x12x1": {"w": 1.0}},
               "digits": {"8": {"w": 1.0}, "7": {"w": 1.2}}}
    rpath = tmp_path / "r.json"
    rpath.write_text(json.dumps(results))
    assert autotune.main(["write", str(rpath), "--header", str(header)]) == 0
    text = header.read_text()
    assert "#define MGPU_SORT_MULTI_THREADS 512" in text
    assert "#define MGPU_SORT_MULTI_ITEMS 12" in text
    assert "#define MGPU_SORT_MAX_DIGIT_BITS 8" in text
    original = open(autotune.CONFIG_H).read()
    for key in ("MGPU_SORT_SINGLE_THREADS", "MGPU_SORT_KEYS_THREADS"):
        line = next(l for l in original.splitlines() if l.startswith(f"#define {key} "))
        assert line in text
    assert text.count("#pragma once") == 1
    # A second write replaces the measurement table instead of stacking it.
    assert autotune.main(["write", str(rpath), "--header", str(header)]) == 0
    assert header.read_text().count("// Measured by the autotuner") == 1


def test_every_candidate_fits_shared_memory():
    """Shared memory of each candidate's largest layout stays within the
    227 KB a B200 CTA may use, and tiles stay below 65536 keys."""
    for cls in ("keys", "single", "multi"):
        for threads, items, _ in autotune.CLASSES[cls]["candidates"]:
            tile = threads * items
            assert tile < 65536
            nw = threads // 32
            if cls == "multi":
                words = tile * (1 + 1 + 6)
            else:
                words = tile * (2 + (0 if cls == "keys" else 1))
            words += nw * 256 + 4 * 256 + 32 + 16
            assert words * 4 <= 227 * 1024, (cls, threads, items)


def test_write_keeps_the_table_of_classes_not_measured(tmp_path):
    header = tmp_path / "tile_config.h"
    shutil.copy(autotune.CONFIG_H, header)
    original = header.read_text()
    assert "//   keys: chosen " in original
    keys_block = [l for l in original.splitlines() if l.startswith("//   keys: chosen ")]
    results = {"small_ballot": {"8": {"w": 1.1}, "5": {"w": 1.0}}}
    rpath = tmp_path / "r.json"
    rpath.write_text(json.dumps(results))
    assert autotune.main(["write", str(rpath), "--header", str(header)]) == 0
    text = header.read_text()
    assert keys_block[0] in text                      # kept
    assert "//   small_ballot: chosen 5" in text       # replaced or added
    assert text.count("//   small_ballot: chosen") == 1
    assert "#define MGPU_SORT_SMALL_BALLOT_BITS 5" in text
    # Classes stay in the autotuner's order.
    order = [c for c in autotune.CLASSES if f"//   {c}: chosen" in text]
    pos = [text.index(f"//   {c}: chosen") for c in order]
    assert pos == sorted(pos)


def test_segmented_check_is_exact():
    """The autotuner's check of segmented results accepts the stable
    per-segment sort and rejects a swap of two equal-key positions."""
    import numpy as np
    import pytest
    case = autotune.make_case("segments_small", 200)
    keys = case.keys.copy()
    keys[::3] &= np.uint32(0xF)                 # many ties
    case.keys = keys
    out_k = np.empty_like(keys)
    out_v = np.empty_like(keys)
    for i in range(case.num_segments):
        a, b = int(case.offsets[i]), int(case.offsets[i + 1])
        o = np.argsort(keys[a:b], kind="stable")
        out_k[a:b] = keys[a:b][o]
        out_v[a:b] = case.values[0][a:b][o]
    autotune.check_segmented(case, out_k, out_v)
    # Two adjacent equal keys of one segment with their positions swapped.
    for i in range(case.num_segments):
        a, b = int(case.offsets[i]), int(case.offsets[i + 1])
        eq = np.flatnonzero(out_k[a + 1:b] == out_k[a:b - 1])
        if eq.size:
            j = a + int(eq[0])
            bad = out_v.copy()
            bad[[j, j + 1]] = bad[[j + 1, j]]
            with pytest.raises(RuntimeError):
                autotune.check_segmented(case, out_k, bad)
            return
    raise AssertionError("no tie found")

"""Autotuner for the sort's tile shapes and digit width (csrc/tile_config.h).

    python -m mgpu_old_b200.autotune build                 # compile every candidate
    python -m mgpu_old_b200.autotune measure -o tune.json  # time them (needs a B200)
    python -m mgpu_old_b200.autotune write tune.json       # rewrite tile_config.h

A candidate is one assignment of tile_config.h's values for one class:
"keys" (keys only), "single" (index mode, one value array), "multi" (two to
six value arrays), "digits" (the widest digit of sortArray's pass plan), or
"<class>_ballot" (how many digit bits the warp ranking of that class resolves
by ballots, the rest by match.any; "small" is the segmented sort's kernel for
segments that fit one tile) or "<class>_batch" (how many items of a thread the
ranking matches before it updates their digit counters). Each
candidate is a separate build of the library (build_variant, under
_build/tune/), because tile shapes are compile-time constants of the
kernels. The build step runs anywhere nvcc does; the measure step loads each
build in its own process, sorts seeded synthetic inputs of the class's
workloads through the C ABI (inputs restored and L2 flushed before each
timed sort, CUDA events around it), checks every result, and records the
median milliseconds. The write step picks, per class, the candidate with
the smallest geometric mean of its time relative to the best candidate on
each workload, and rewrites tile_config.h with the winners and a table of
the measurements.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CONFIG_H = os.path.join(HERE, "csrc", "tile_config.h")

CLASSES = {
    "keys": {
        "keys": ("MGPU_SORT_KEYS_THREADS", "MGPU_SORT_KEYS_ITEMS", "MGPU_SORT_KEYS_MIN_BLOCKS"),
        "candidates": [(384, 20, 2), (512, 14, 2), (512, 16, 2), (384, 24, 2), (256, 20, 3)],
        "workloads": [("keys_u32", 1 << 20), ("keys_u32", 1 << 24), ("keys_u32", 1 << 26)],
    },
    # Keys-only passes of MGPU_SORT_KEYS_LARGE_ELEMENTS keys or more.
    "keys_large": {
        "keys": ("MGPU_SORT_KEYS_LARGE_THREADS", "MGPU_SORT_KEYS_LARGE_ITEMS",
                 "MGPU_SORT_KEYS_LARGE_MIN_BLOCKS"),
        "candidates": [(256, 28, 3), (256, 20, 3), (256, 32, 2), (512, 14, 2), (384, 20, 2)],
        "workloads": [("keys_u32", 1 << 25), ("keys_u32", 1 << 26), ("keys_u32", 3 << 25)],
    },
    "single": {
        "keys": ("MGPU_SORT_SINGLE_THREADS", "MGPU_SORT_SINGLE_ITEMS",
                 "MGPU_SORT_SINGLE_MIN_BLOCKS"),
        "candidates": [(256, 32, 2), (256, 30, 2), (384, 20, 2), (256, 20, 3), (512, 14, 2),
                       (384, 16, 2), (256, 24, 2), (768, 10, 1)],
        "workloads": [("pairs_and24", 1 << 25), ("pairs_u32", 1 << 26), ("index_u32", 1 << 24)],
    },
    # The segmented sort's range passes with index mode or one value array.
    "seg_single": {
        "keys": ("MGPU_SORT_SEG_SINGLE_THREADS", "MGPU_SORT_SEG_SINGLE_ITEMS",
                 "MGPU_SORT_SEG_SINGLE_MIN_BLOCKS"),
        "candidates": [(384, 20, 2), (256, 32, 2), (512, 14, 2), (256, 24, 2)],
        "workloads": [("segments_lognormal", 10_000)],
    },
    "multi": {
        "keys": ("MGPU_SORT_MULTI_THREADS", "MGPU_SORT_MULTI_ITEMS",
                 "MGPU_SORT_MULTI_MIN_BLOCKS"),
        "candidates": [(768, 8, 1), (512, 12, 1), (576, 10, 1), (384, 16, 1)],
        "workloads": [("multi6_17bit", 1 << 24), ("multi3_u32", 1 << 24)],
    },
    "digits": {
        "keys": ("MGPU_SORT_MAX_DIGIT_BITS",),
        "candidates": [(8,), (7,), (6,)],
        "workloads": [("pairs_and24", 1 << 25), ("keys_u32", 1 << 24)],
    },
    # How the warp ranking finds the lanes sharing a digit: ballots on the
    # low 8, 5 or 4 digit bits, match.any on the rest (match_digit8).
    "keys_ballot": {
        "keys": ("MGPU_SORT_KEYS_BALLOT_BITS",),
        "candidates": [(8,), (5,), (4,)],
        "workloads": [("keys_u32", 1 << 24), ("keys_u32", 1 << 26)],
    },
    "single_ballot": {
        "keys": ("MGPU_SORT_SINGLE_BALLOT_BITS",),
        "candidates": [(8,), (5,), (4,)],
        "workloads": [("pairs_and24", 1 << 25), ("pairs_u32", 1 << 24), ("index_u32", 1 << 24),
                      ("segments_lognormal", 10_000)],
    },
    # The same choice for sortArray calls of MGPU_SORT_SINGLE_LARGE_ELEMENTS
    # keys or more.
    "single_large_ballot": {
        "keys": ("MGPU_SORT_SINGLE_LARGE_BALLOT_BITS",),
        "candidates": [(8,), (5,), (4,)],
        "workloads": [("pairs_u32", 1 << 26), ("pairs_u32", 3 << 25), ("index_u32", 1 << 26)],
    },
    "multi_ballot": {
        "keys": ("MGPU_SORT_MULTI_BALLOT_BITS",),
        "candidates": [(8,), (5,), (4,)],
        "workloads": [("multi6_17bit", 1 << 24), ("multi3_u32", 1 << 24)],
    },
    # Items per thread whose peers are found before the counter updates.
    "keys_batch": {
        "keys": ("MGPU_SORT_KEYS_RANK_BATCH",),
        "candidates": [(1,), (4,), (5,), (10,), (20,)],
        "workloads": [("keys_u32", 1 << 24), ("keys_u32", 1 << 26)],
    },
    "single_batch": {
        "keys": ("MGPU_SORT_SINGLE_RANK_BATCH",),
        "candidates": [(1,), (4,), (5,), (8,), (10,), (16,), (20,)],
        "workloads": [("pairs_and24", 1 << 25), ("pairs_u32", 1 << 26), ("index_u32", 1 << 24),
                      ("segments_lognormal", 10_000)],
    },
    "multi_batch": {
        "keys": ("MGPU_SORT_MULTI_RANK_BATCH",),
        "candidates": [(1,), (2,), (4,), (8,)],
        "workloads": [("multi6_17bit", 1 << 24), ("multi3_u32", 1 << 24)],
    },
    "small_batch": {
        "keys": ("MGPU_SORT_SMALL_RANK_BATCH",),
        "candidates": [(1,), (2,), (4,), (8,), (16,)],
        "workloads": [("segments_small", 50_000)],
    },
    "small_ballot": {
        "keys": ("MGPU_SORT_SMALL_BALLOT_BITS",),
        "candidates": [(8,), (5,), (4,)],
        "workloads": [("segments_small", 50_000)],
    },
}


def variant_name(cls: str, values: tuple) -> str:
    return cls + "_" + "x".join(str(v) for v in values)


def defines(cls: str, values: tuple) -> dict:
    return dict(zip(CLASSES[cls]["keys"], values))


def cmd_build(args) -> int:
    from concurrent.futures import ThreadPoolExecutor
    from mgpu_old_b200 import build
    jobs = [(cls, values) for cls, spec in CLASSES.items()
            if not args.only or cls in args.only for values in spec["candidates"]]

    def one(job):
        cls, values = job
        name = variant_name(cls, values)
        try:
            return f"built {name}: {build.build_variant(name, defines(cls, values))}"
        except subprocess.CalledProcessError:
            return f"skipped {name}: does not build"

    with ThreadPoolExecutor(max_workers=args.jobs) as pool:
        for line in pool.map(one, jobs):
            print(line, flush=True)
    return 0


def make_case(kind: str, n: int):
    from mgpu_old_b200 import workloads
    if kind == "pairs_and24":
        return workloads.pairs_and24(n)
    if kind == "pairs_u32":
        return workloads.pairs_uniform32(n)
    if kind == "keys_u32":
        return workloads.keys_uniform32(n, seed=6)
    if kind == "index_u32":
        c = workloads.keys_uniform32(n, seed=8)
        c.value_count = -1
        return c
    if kind == "multi6_17bit":
        return workloads.multi6_17bit(n)
    if kind == "segments_lognormal":
        return workloads.segments_lognormal(n)
    if kind == "segments_small":
        # Many short segments (median 256): the small-segment kernel's work.
        import numpy as np
        sizes = np.clip(np.rint(np.random.default_rng(12).lognormal(np.log(256.0), 1.0, n)),
                        1, 4096).astype(np.int64)
        offsets = np.zeros(n + 1, np.int64)
        np.cumsum(sizes, out=offsets[1:])
        total = int(offsets[-1])
        keys = np.random.default_rng(13).integers(0, 1 << 32, total, dtype=np.uint64)
        local = (np.arange(total, dtype=np.int64) - np.repeat(offsets[:-1], sizes))
        return workloads.SegmentedCase(f"segments_small_{n}", keys.astype(np.uint32),
                                       [local.astype(np.uint32)], 1, 0, 32,
                                       offsets=offsets.astype(np.int32))
    if kind == "multi3_u32":
        import numpy as np
        rng = np.random.Generator(np.random.MT19937(9))
        keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        vals = [np.arange(n, dtype=np.uint32)] + \
            [rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32) for _ in range(2)]
        return workloads.SortCase(f"multi3_u32_{n}", keys, vals, 3, 0, 32)
    raise ValueError(kind)


def check_segmented(case, keys, local) -> None:
    """Exact check of a segmented sort whose value array holds each key's
    position within its segment: every segment's keys are its input keys
    ordered stably (ties keep input order)."""
    import numpy as np
    sizes = np.diff(case.offsets.astype(np.int64))
    seg = np.repeat(np.arange(sizes.size), sizes)
    order = np.lexsort((case.keys, seg))      # stable within equal keys
    if not np.array_equal(keys, case.keys[order]):
        raise RuntimeError(f"{case.name}: keys differ from a stable per-segment sort")
    start = case.offsets[:-1].astype(np.int64)
    if not np.array_equal(local.astype(np.int64) + np.repeat(start, sizes), order):
        raise RuntimeError(f"{case.name}: positions differ from a stable per-segment sort")


def time_segmented(case, steps: int) -> float:
    """Median ms of `steps` sortSegmentedArray calls on the case, after an
    exact check of the result."""
    import numpy as np
    import torch
    from mgpu_old_b200 import api
    dev = torch.device("cuda", 0)
    n = case.n
    cap = (n + 2047) // 2048 * 2048
    src_k = torch.zeros(cap, dtype=torch.int32, device=dev)
    src_v = torch.zeros(cap, dtype=torch.int32, device=dev)
    src_k[:n] = torch.from_numpy(case.keys.view(np.int32)).to(dev)
    src_v[:n] = torch.from_numpy(case.values[0].view(np.int32)).to(dev)
    offs = torch.from_numpy(case.offsets.astype(np.int32)).to(dev)
    k = [torch.empty(cap, dtype=torch.int32, device=dev) for _ in range(2)]
    v = [torch.empty(cap, dtype=torch.int32, device=dev) for _ in range(2)]
    d = api.SortData()
    d.maxElements, d.numElements, d.valueCount = cap, n, 1
    d.firstBit, d.endBit = case.first_bit, case.end_bit
    d.keys[0], d.keys[1] = k[0].data_ptr(), k[1].data_ptr()
    d.values[0][0], d.values[0][1] = v[0].data_ptr(), v[1].data_ptr()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    eng = api.MgpuSort()
    times = []
    for it in range(steps + 3):
        k[0].copy_(src_k)
        v[0].copy_(src_v)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        api.check(eng.sort_segmented(d, offs.data_ptr(), case.num_segments))
        e1.record()
        e1.synchronize()
        if it >= 3:
            times.append(e0.elapsed_time(e1))
    api.check(eng.synchronize())
    check_segmented(case, k[0][:n].cpu().numpy().view(np.uint32),
                    v[0][:n].cpu().numpy().view(np.uint32))
    eng.release()
    return sorted(times)[len(times) // 2]


def time_case(case, steps: int) -> float:
    """Median ms of `steps` sorts of the case through sortArray, after a
    check of the result (the first value array, when it holds the input
    positions, must gather the input keys into the sorted output)."""
    from mgpu_old_b200 import workloads
    if isinstance(case, workloads.SegmentedCase):
        return time_segmented(case, steps)
    import numpy as np
    import torch
    from mgpu_old_b200 import api
    dev = torch.device("cuda", 0)
    n = case.n
    cap = (n + 2047) // 2048 * 2048
    arrays = 1 if case.value_count == -1 else case.value_count

    def buf(a=None):
        t = torch.empty(cap, dtype=torch.int32, device=dev)
        if a is not None:
            t[:n] = torch.from_numpy(a.view(np.int32)).to(dev)
        return t

    src_k = buf(case.keys)
    src_v = [buf(v) for v in case.values]
    bufs = {}
    d = api.SortData()
    d.maxElements, d.numElements, d.valueCount = cap, n, case.value_count
    d.firstBit, d.endBit = case.first_bit, case.end_bit
    for j in range(2):
        t = buf()
        bufs[t.data_ptr()] = t
        d.keys[j] = t.data_ptr()
    for i in range(arrays):
        for j in range(2):
            t = buf()
            bufs[t.data_ptr()] = t
            d.values[i][j] = t.data_ptr()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    eng = api.MgpuSort()

    def restore():
        bufs[d.keys[0]][:n].copy_(src_k[:n])
        for i, v in enumerate(src_v):
            bufs[d.values[i][0]][:n].copy_(v[:n])

    times = []
    for it in range(steps + 3):
        restore()
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        api.check(eng.sort_array(d))
        e1.record()
        e1.synchronize()
        if it >= 3:
            times.append(e0.elapsed_time(e1))
    api.check(eng.synchronize())
    keys = bufs[d.keys[0]][:n].cpu().numpy().view(np.uint32)
    bits = case.end_bit - case.first_bit
    mask = np.uint32(0xFFFFFFFF if bits >= 32 else (1 << bits) - 1)
    field = (keys >> np.uint32(case.first_bit)) & mask
    if (np.diff(field.astype(np.int64)) < 0).any():
        raise RuntimeError(f"{case.name}: output not sorted")
    if case.value_count == -1 or (case.value_count >= 1 and np.array_equal(
            case.values[0][:16], np.arange(16, dtype=np.uint32))):
        idx = bufs[d.values[0][0]][:n].cpu().numpy().view(np.uint32)
        if not np.array_equal(keys, case.keys[idx]):
            raise RuntimeError(f"{case.name}: values do not follow the keys")
    eng.release()
    return sorted(times)[len(times) // 2]


def cmd_time(args) -> int:
    """Child process: one build, one class's workloads; prints JSON."""
    import torch
    from mgpu_old_b200 import api
    api.load_library(args.lib)
    torch.cuda.set_device(0)
    out = {}
    for kind, n in CLASSES[args.cls]["workloads"]:
        out[f"{kind}_{n}"] = time_case(make_case(kind, n), args.steps)
    print(json.dumps(out))
    return 0


def cmd_measure(args) -> int:
    from mgpu_old_b200 import build
    results = {}
    for cls, spec in CLASSES.items():
        if args.only and cls not in args.only:
            continue
        results[cls] = {}
        for values in spec["candidates"]:
            name = variant_name(cls, values)
            lib = os.path.join(HERE, "_build", "tune", name, build.LIB_NAME)
            if not os.path.exists(lib):
                print(f"{name}: not built", file=sys.stderr)
                continue
            p = subprocess.run([sys.executable, "-m", "mgpu_old_b200.autotune", "_time", lib,
                                cls, "--steps", str(args.steps)],
                               capture_output=True, text=True, cwd=os.path.dirname(HERE))
            if p.returncode != 0:
                print(f"{name}: failed\n{p.stderr[-2000:]}", file=sys.stderr)
                continue
            results[cls]["x".join(map(str, values))] = json.loads(p.stdout.strip().splitlines()[-1])
            print(name, results[cls]["x".join(map(str, values))], flush=True)
    with open(args.output, "w") as f:
        json.dump(results, f, indent=1)
    return 0


def choose(table: dict) -> tuple[str, dict]:
    """The candidate with the smallest geometric mean of time relative to
    the best candidate per workload; also every candidate's score."""
    workloads = sorted({w for t in table.values() for w in t})
    best = {w: min(t[w] for t in table.values() if w in t) for w in workloads}
    scores = {}
    for cand, t in table.items():
        if all(w in t for w in workloads):
            scores[cand] = math.exp(sum(math.log(t[w] / best[w]) for w in workloads)
                                    / len(workloads))
    winner = min(scores, key=scores.get)
    return winner, scores


def cmd_write(args) -> int:
    with open(args.results) as f:
        results = json.load(f)
    header = args.header or CONFIG_H
    with open(header) as f:
        text = f.read()
    import re
    # The table already in the header, one block of lines per class: blocks
    # of classes measured again are replaced, the others kept.
    blocks = {}
    start = text.find("// Measured by the autotuner")
    if start >= 0:
        end = text.find("#pragma once")
        cls = None
        for line in text[start:end].splitlines():
            m = re.match(r"//   (\w+): chosen ", line)
            if m:
                cls = m.group(1)
                blocks[cls] = []
            if cls:
                blocks[cls].append(line)
        text = text[:start] + text[end:]
    for cls, table in results.items():
        if not table:
            continue
        winner, scores = choose(table)
        for key, val in zip(CLASSES[cls]["keys"], winner.split("x")):
            text = re.sub(rf"#define {key} \d+", f"#define {key} {val}", text)
        lines = [f"//   {cls}: chosen {winner}"]
        for cand, t in sorted(table.items(), key=lambda kv: scores.get(kv[0], 9)):
            cells = ", ".join(f"{w} {ms:.3f}" for w, ms in sorted(t.items()))
            lines.append(f"//     {cand:>10}  score {scores.get(cand, float('nan')):.3f}  "
                         f"{cells}")
        blocks[cls] = lines
    table_lines = ["// Measured by the autotuner (median ms per sort; score = geometric",
                   "// mean of time / best time over the class's workloads):"]
    for cls in CLASSES:
        table_lines += blocks.pop(cls, [])
    for lines in blocks.values():
        table_lines += lines
    text = text.replace("#pragma once", "\n".join(table_lines) + "\n#pragma once", 1)
    with open(header, "w") as f:
        f.write(text)
    print(f"wrote {header}")
    return 0


def main(argv=None) -> int:
    p = argparse.ArgumentParser()
    sub = p.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("build")
    b.add_argument("--only", nargs="*")
    b.add_argument("--jobs", type=int, default=4)
    m = sub.add_parser("measure")
    m.add_argument("-o", "--output", default="tune.json")
    m.add_argument("--steps", type=int, default=7)
    m.add_argument("--only", nargs="*")
    w = sub.add_parser("write")
    w.add_argument("results")
    w.add_argument("--header", default=None, help="file to rewrite (default: tile_config.h)")
    t = sub.add_parser("_time")
    t.add_argument("lib")
    t.add_argument("cls")
    t.add_argument("--steps", type=int, default=7)
    args = p.parse_args(argv)
    return {"build": cmd_build, "measure": cmd_measure, "write": cmd_write,
            "_time": cmd_time}[args.cmd](args)


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark of the sortArray path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl ours|reference]

A step is one sortArray call over one batch of synthetic input (default:
67,108,864 uint32 key + value pairs, keys uniform over 32 bits, value =
index, bits [0, 32): the 64M-pair target configuration). Each timed step
starts from freshly restored input and a flushed L2 (a 256 MiB write between
steps; the restore copy and the flush are outside the timed region). `value`
is device-resident throughput in Mkeys/s over the K timed steps (CUDA events
on the sort's stream, max over ranks); `e2e` is the same metric through the C
ABI with pinned host buffers, host->device and device->host copies inside the
timed region, beside the bound that the copies alone set (`e2e.copy_bound`).
The roofline entry is the sort kernel of a pass (the dominant kernel), whose
launches are timed with CUDA events around each launch in a second run of the
same timed steps (sortEnableKernelTiming), so that the events do not slow the
run that gives `value`.

Multi-GPU: the sort path does not shard (one global order), so N ranks run N
independent replicas of the workload ("weak" scaling); the only collectives
are the barrier and the max-over-ranks of the timings.

--impl reference times the reference's CPU sort path on this host over the
whole workload per step: for keys-only uint32 workloads the reference's own
sort/src/cpusort/cpusort.cpp compiled from its source (oracle/_ref), else the
oracle's restatement of its algorithm (cpusort.cpp:122-186) extended to value
arrays, on all host threads. That arm never loads the library.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mgpu_old_b200 import workloads  # noqa: E402

METRIC = "sort Mkeys/s"
UNIT = "Mkeys/s"
FALLBACK_HBM_GBS = 6650.0
CPU_SAMPLE = 1 << 22


# Batches in flight in the end-to-end measurement (one engine, stream and
# set of device buffers each).
E2E_LANES = 3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="pairs_u32_64M",
                   choices=sorted(workloads.WORKLOADS) + ["served", "bwt"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--server-slots", type=int, default=4,
                   help="served workload: server slots (engine + stream each)")
    p.add_argument("--bwt-bytes", type=int, default=8 << 20,
                   help="bwt workload: block size in bytes")
    p.add_argument("--bwt-key", type=int, default=16,
                   help="bwt workload: gpuKeySize (symbols ordered on the GPU)")
    p.add_argument("--requests", type=int, default=2000,
                   help="served workload: number of requests")
    p.add_argument("--server-budget", type=int, default=64,
                   help="served workload: device memory budget in GiB")
    p.add_argument("--profile-only", action="store_true",
                   help="warm-up plus --steps sorts, no e2e/CPU legs (for ncu)")
    return p.parse_args()


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload_config(case, args, extra=None):
    cfg = {"workload": case.name, "n": case.n, "value_count": case.value_count,
           "first_bit": case.first_bit, "end_bit": case.end_bit,
           "passes": len(_plan(case)), "parallelism": f"replicas{args.gpus}",
           "l2": "flushed between steps (256 MiB write); inputs restored between steps"}
    if extra:
        cfg.update(extra)
    return cfg


def _plan(case):
    """sortArray's pass widths over the case's bit range: ceil(bits / 8)
    passes, widths balanced. Plain Python, so that the CPU arms never load the
    library."""
    bits = case.end_bit - case.first_bit
    p = (bits + 7) // 8
    return [bits // p + (i < bits % p) for i in range(p)]


# ---------------------------------------------------------------------------
# The BWT caller (include/mgpubwt.h): block sort of an English-like text block.

BWT_METRIC = "bwtSortBlock MB/s"
BWT_CPU_SAMPLE = 1 << 20


def bwt_config(args, extra=None):
    cfg = {"workload": "bwt_text", "block_bytes": args.bwt_bytes, "gpu_key_size": args.bwt_key,
           "block": "seeded English-like text (500-word Zipf vocabulary)",
           "parallelism": f"replicas{args.gpus}"}
    if extra:
        cfg.update(extra)
    return cfg


def cpu_bwt_sample(block):
    """Seconds of one host block sort of `block`: the reference BWT library's
    own string quicksort (bwt/src/mgpubwt/cpusort.cpp, built in oracle/_ref)
    when present, else the oracle's stable sort of rotations."""
    from oracle import oracle
    oracle.build(ref=False)
    t0 = time.perf_counter()
    if oracle.ref_bwt_lib() is not None:
        oracle.ref_bwt_block(block)
        kind = "reference"
    else:
        oracle.bwt(block, 1)
        kind = "port"
    return time.perf_counter() - t0, kind


def cpu_baseline_bwt(args, budget_s=10.0):
    block = workloads.text_block(min(args.bwt_bytes, BWT_CPU_SAMPLE))
    total_t, reps, kind = 0.0, 0, "port"
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end or reps == 0:
        t, kind = cpu_bwt_sample(block)
        total_t += t
        reps += 1
    what = ("the reference's QSortStrings (bwt/src/mgpubwt/cpusort.cpp) over every rotation"
            if kind == "reference" else "the oracle's stable sort of rotations")
    return {"value": round(block.size * reps / total_t / 1e6, 3), "unit": "MB/s", "cores": 1,
            "kind": kind, "sample": f"{block.size}-byte block of the same text, {what}, "
                                    f"1 thread, {reps} repetitions"}


def run_bwt(args, barrier, max_over_ranks, world, rank, local=0):
    """bwtSortBlock on a host block (its API takes and returns host memory),
    wall clock around each synchronous call; every result is checked against
    the oracle's rotation sort once."""
    from mgpu_old_b200 import api
    from oracle import oracle
    block = workloads.text_block(args.bwt_bytes)
    eng = api.BwtEngine()
    for _ in range(max(args.warmup, 3)):
        st, idx, xf, seg, av = eng.sort_block(block, args.bwt_key)
        if st != api.BwtStatus.SUCCESS:
            raise SystemExit(f"bwtSortBlock: {api.bwt_status_string(st)}")
    e_idx, e_xf, e_seg, _ = oracle.bwt(block, args.bwt_key)
    if not (np.array_equal(idx, e_idx) and np.array_equal(xf, e_xf) and seg == e_seg):
        raise SystemExit("bwt result differs from the oracle")
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        eng.sort_block(block, args.bwt_key)
        times.append(time.perf_counter() - t0)
    clk = clocks.stop()
    ms = max_over_ranks(sum(times) / len(times) * 1e3)
    value = block.size * world / (ms * 1e-3) / 1e6
    eng.close()
    line = {"metric": BWT_METRIC, "value": round(value, 2), "unit": "MB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded numpy)",
            "config": bwt_config(args, {"tie_groups": seg, "mean_tie_group": round(av, 3),
                                        "timing": "wall clock around the synchronous host call"}),
            "e2e": {"value": round(value, 2), "unit": "MB/s",
                    "h2d_bytes_per_step": 2 * block.size + 32,
                    "d2h_bytes_per_step": 5 * block.size},
            "clocks": clk}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_bwt(args)
    return line


def run_reference_bwt(args):
    """Reference arm for the BWT caller: the reference's host block sort
    (QSortStrings over every rotation, as its TinyBlockSort) on a bounded
    1 MiB block of the same text per step."""
    block = workloads.text_block(min(args.bwt_bytes, BWT_CPU_SAMPLE))
    for _ in range(args.warmup):
        cpu_bwt_sample(block)
    runs = [cpu_bwt_sample(block) for _ in range(args.steps)]
    total = sum(t for t, _ in runs)
    kind = runs[-1][1]
    value = block.size * len(runs) / total / 1e6
    line = {"impl": "reference", "metric": BWT_METRIC, "value": round(value, 3), "unit": "MB/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total / len(runs) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": bwt_config(args, {"sample_bytes": block.size}),
            "cpu_baseline": {"value": round(value, 3), "unit": "MB/s", "cores": 1, "kind": kind,
                             "sample": f"{block.size}-byte block per step"},
            "e2e": {"value": round(value, 3), "unit": "MB/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# CPU side. The reference's CPU sort (sort/src/cpusort/cpusort.cpp) sorts keys
# only: for keys-only workloads its own code, compiled from its source into
# oracle/_ref, is timed ("reference"); where values ride along, the oracle's
# LSD restatement of the same algorithm (cpusort.cpp:122-186, extended to
# value arrays and bit ranges, its per-block phases on all host threads) is
# timed instead ("port").


def _lsd_full(case, threads):
    """The oracle's LSD sort of the whole workload on `threads` host threads.
    Returns (seconds, keys, values)."""
    from oracle import oracle
    oracle.build(ref=False)
    t0 = time.perf_counter()
    keys = case.keys
    if case.key_type:
        keys = workloads.key_image(keys, case.key_type)
    k, v = oracle.sort_lsd(keys, case.values, case.value_count, case.first_bit,
                           _plan(case), 1 << 15, threads)
    if case.key_type:
        k = workloads.key_preimage(k, case.key_type)
    return time.perf_counter() - t0, k, v


def _ref_sort2_usable(case):
    """The reference's own CPU sort handles this workload: uint32 keys only."""
    if case.value_count != 0 or case.key_type:
        return False
    from oracle import oracle
    return oracle.ref_lib() is not None


def _ref_sort2(case):
    """The reference's CPU radix sort (cpusort.cpp Sort2Pass, blocked 4-bit
    passes as its Sort2 makes them, sequential as written) over the case's
    bit range. Returns (seconds, keys)."""
    from oracle import oracle
    ref = oracle.ref_lib()
    k = np.array(case.keys, dtype=np.uint32, copy=True)
    t0 = time.perf_counter()
    bit = case.first_bit
    while bit < case.end_bit:
        nb = min(4, case.end_bit - bit)
        ref.ref_cpusort_sort2pass(oracle._p(k), bit, nb, k.size, 2048)
        bit += nb
    return time.perf_counter() - t0, k


def _stable_sample(case, sample_n):
    """std::stable_sort by the bit field (the oracle's stable leg) on one
    core over the first sample_n elements. Returns seconds."""
    from oracle import oracle
    oracle.build(ref=False)
    keys = np.ascontiguousarray(case.keys[:sample_n])
    if case.key_type:
        keys = workloads.key_image(keys, case.key_type)
    vals = [np.ascontiguousarray(v[:sample_n]) for v in case.values]
    t0 = time.perf_counter()
    oracle.sort_stable(keys, vals, case.value_count, case.first_bit, case.end_bit)
    return time.perf_counter() - t0


def cpu_baseline(case, gpu_keys, gpu_vals, budget_s=20.0):
    """Times the CPU path on the host cores over the whole workload and, as
    the checker, compares the GPU result with its output bit for bit (keys
    and every value array). Also reports std::stable_sort on one core over a
    bounded sample and, for keys-only workloads, the reference's own Sort2."""
    threads = os.cpu_count() or 1
    t, k, v = _lsd_full(case, threads)
    if not np.array_equal(k, gpu_keys):
        raise AssertionError("GPU keys differ from the oracle")
    for i, (a, b) in enumerate(zip(gpu_vals, v)):
        if not np.array_equal(a, b):
            raise AssertionError(f"GPU value array {i} differs from the oracle")
    times = [t]
    t_end = time.perf_counter() + budget_s / 2
    while time.perf_counter() < t_end and len(times) < 5:
        times.append(_lsd_full(case, threads)[0])
    lsd_t = min(times)
    out = {"value": round(case.n / lsd_t / 1e6, 3), "unit": UNIT, "cores": threads,
           "kind": "port",
           "sample": f"the whole workload ({case.n} elements, all value arrays), oracle LSD "
                     f"radix (cpusort.cpp:122-186 restated, 8-bit passes) on {threads} "
                     f"threads, best of {len(times)}",
           "oracle_check": "GPU keys and every value array equal the oracle's, bit for bit"}
    sample_n = min(case.n, CPU_SAMPLE)
    st = _stable_sample(case, sample_n)
    out["std_stable_sort"] = {"value": round(sample_n / st / 1e6, 3), "unit": UNIT, "cores": 1,
                              "sample": f"first {sample_n} elements, std::stable_sort of "
                                        "positions by the bit field, values gathered"}
    if _ref_sort2_usable(case):
        rt, rk = _ref_sort2(case)
        if not np.array_equal(rk, gpu_keys):
            raise AssertionError("GPU keys differ from the reference's own CPU sort")
        out["reference_sort2"] = {"value": round(case.n / rt / 1e6, 3), "unit": UNIT,
                                  "cores": 1, "kind": "reference",
                                  "sample": "the whole workload, cpusort.cpp Sort2Pass "
                                            "4-bit passes built from the reference source"}
    return out


def cpu_baseline_segmented(case, budget_s=10.0):
    """The oracle's per-segment stable sort on a bounded sample of segments."""
    from oracle import oracle
    oracle.build(ref=False)
    sizes = np.diff(case.offsets.astype(np.int64))
    take = int(np.searchsorted(np.cumsum(sizes), CPU_SAMPLE)) + 1
    take = max(1, min(take, case.num_segments))
    end = int(case.offsets[take])
    offs = case.offsets[:take + 1]
    keys = case.keys[:end]
    vals = [case.values[0][:end]]
    total_t, total_n = 0.0, 0
    t_end = time.perf_counter() + budget_s
    while time.perf_counter() < t_end or total_n == 0:
        t0 = time.perf_counter()
        oracle.sort_segments(keys, vals, 1, offs, case.first_bit, case.end_bit)
        total_t += time.perf_counter() - t0
        total_n += end
    return {"value": round(total_n / total_t / 1e6, 3), "unit": UNIT, "cores": 1,
            "kind": "port",
            "sample": f"first {take} segments ({end} elements) of {case.name}, oracle "
                      f"std::stable_sort per segment, 1 thread, {total_n // end} repetitions"}


def run_reference_segmented(args, case):
    """Reference arm for a segmented workload: the oracle's per-segment
    stable sort (what a per-segment loop of the CPU path computes) over a
    bounded sample of segments per step."""
    from oracle import oracle
    oracle.build(ref=False)
    sizes = np.diff(case.offsets.astype(np.int64))
    take = max(1, min(case.num_segments, int(np.searchsorted(np.cumsum(sizes), CPU_SAMPLE)) + 1))
    end = int(case.offsets[take])
    offs, keys, vals = case.offsets[:take + 1], case.keys[:end], [case.values[0][:end]]
    for _ in range(args.warmup):
        oracle.sort_segments(keys, vals, 1, offs, case.first_bit, case.end_bit)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.sort_segments(keys, vals, 1, offs, case.first_bit, case.end_bit)
        times.append(time.perf_counter() - t0)
    value = end * len(times) / sum(times) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(sum(times) / len(times) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(case, args, {"sample_segments": take, "sample": end}),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"first {take} segments per step"},
            "e2e": {"value": round(value, 3), "unit": UNIT,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference_served(args):
    """Reference arm for the served workload: the oracle's multithreaded LSD
    sort (cpusort.cpp:122-186 restated) of each request in arrival order, over
    a bounded sample of requests per step."""
    from oracle import oracle
    oracle.build(ref=False)
    sizes, has_values, end_bits, rng = served_requests(args.requests)
    threads = os.cpu_count() or 1
    take = max(1, int(np.searchsorted(np.cumsum(sizes), CPU_SAMPLE)))
    pool = rng.integers(0, 1 << 32, int(sizes[:take].max()), dtype=np.uint64).astype(np.uint32)
    idx = np.arange(pool.size, dtype=np.uint32)

    def one_step():
        t0 = time.perf_counter()
        for i in range(take):
            n, end = int(sizes[i]), int(end_bits[i])
            p = (end + 7) // 8
            widths = [end // p + (j < end % p) for j in range(p)]
            vals = [idx[:n]] if has_values[i] else []
            oracle.sort_lsd(pool[:n], vals, 1 if has_values[i] else 0, 0, widths, 1 << 15,
                            threads)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        one_step()
    times = [one_step() for _ in range(args.steps)]
    elems = int(sizes[:take].sum())
    value = elems * len(times) / sum(times) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(sum(times) / len(times) * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "served_requests", "sample_requests": take,
                       "sample": elems},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads,
                             "kind": "port", "sample": f"first {take} requests per step"},
            "e2e": {"value": round(value, 3), "unit": UNIT,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference(args):
    """Reference arm: the reference's CPU sort path over the whole workload
    per step, on this host's cores. Keys-only uint32 workloads run the
    reference's own cpusort.cpp (Sort2Pass, compiled from its source into
    oracle/_ref; sequential code, one thread); workloads with value arrays
    run the oracle's restatement of it extended to values, on all host
    threads. Warm-up is capped at one step and the timed steps at a time
    budget, so that the arm ends within a few minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "served":
        return run_reference_served(args)
    if args.workload == "bwt":
        return run_reference_bwt(args)
    case = workloads.WORKLOADS[args.workload]()
    if isinstance(case, workloads.SegmentedCase):
        return run_reference_segmented(args, case)
    threads = os.cpu_count() or 1
    if _ref_sort2_usable(case):
        kind, cores = "reference", 1
        what = "cpusort.cpp Sort2Pass (blocked 4-bit passes) built from the reference source"

        def step():
            return _ref_sort2(case)[0]
    else:
        kind, cores = "port", threads
        what = (f"oracle LSD radix (cpusort.cpp:122-186 restated with value arrays, 8-bit "
                f"passes) on {threads} threads")

        def step():
            return _lsd_full(case, threads)[0]
    for _ in range(min(args.warmup, 1)):
        step()
    budget_s = 150.0
    t_end = time.perf_counter() + budget_s
    times = []
    for _ in range(args.steps):
        times.append(step())
        if time.perf_counter() > t_end:
            break
    total = sum(times)
    value = case.n * len(times) / total / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "steps_timed": len(times),
            "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded numpy MT19937)",
            "config": workload_config(case, args),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores,
                             "kind": kind,
                             "sample": f"the whole workload per step ({case.n} elements), "
                                       f"{what}"},
            "e2e": {"value": round(value, 3), "unit": UNIT,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU side


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        """Start sampling; returns once the first sample arrived (or 10 s)."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
            return
        t_end = time.time() + 10
        while not self.lines and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.02)
        self.first = len(self.lines)

    def wait_one_more(self):
        """Block until at least one sample was taken after start()."""
        t_end = time.time() + 5
        while self.proc and len(self.lines) <= getattr(self, "first", 0) \
                and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.wait_one_more()
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines[max(getattr(self, "first", 1) - 1, 0):]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class GpuSorter:
    """Device buffers for one workload plus a pristine copy to restore from."""

    def __init__(self, case, device):
        import torch
        from mgpu_old_b200 import api
        self.api = api
        self.case = case
        self.n = case.n
        cap = (self.n + 2047) // 2048 * 2048
        self.arrays = 1 if case.value_count == -1 else case.value_count

        def dev(a):
            t = torch.empty(cap, dtype=torch.int32, device=device)
            t[:self.n] = torch.from_numpy(a.view(np.int32)).to(device)
            return t

        self.src_keys = dev(case.keys)
        self.src_vals = [dev(v) for v in case.values]
        self.bufs = {}
        d = api.SortData()
        d.maxElements, d.numElements, d.valueCount = cap, self.n, case.value_count
        d.firstBit, d.endBit = case.first_bit, case.end_bit
        for j in range(2):
            t = torch.empty(cap, dtype=torch.int32, device=device)
            self.bufs[t.data_ptr()] = t
            d.keys[j] = t.data_ptr()
        for i in range(self.arrays):
            for j in range(2):
                t = torch.empty(cap, dtype=torch.int32, device=device)
                self.bufs[t.data_ptr()] = t
                d.values[i][j] = t.data_ptr()
        self.data = d
        self.flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=device)

    def restore(self):
        d = self.data
        self.bufs[d.keys[0]][:self.n].copy_(self.src_keys[:self.n])
        for i in range(len(self.src_vals)):
            self.bufs[d.values[i][0]][:self.n].copy_(self.src_vals[i][:self.n])

    def flush_l2(self):
        self.flush_buf.zero_()

    def result(self):
        d = self.data
        keys = self.bufs[d.keys[0]][:self.n].cpu().numpy().view(np.uint32)
        vals = [self.bufs[d.values[i][0]][:self.n].cpu().numpy().view(np.uint32)
                for i in range(self.arrays)]
        return keys, vals


def verify(case, keys, vals):
    """Cheap full-size checks: field order, key multiset, and for index-valued
    workloads the exact stable permutation."""
    bits = case.end_bit - case.first_bit
    mask = np.uint32(0xFFFFFFFF if bits >= 32 else (1 << bits) - 1)
    f = (workloads.key_image(keys, case.key_type) >> np.uint32(case.first_bit)) & mask
    assert (f[1:] >= f[:-1]).all(), "output not ordered"
    assert np.array_equal(np.sort(keys), np.sort(case.keys)), "keys not a permutation"
    if case.value_count == 1 and np.array_equal(case.values[0][:16], np.arange(16)):
        idx = vals[0]
        assert np.array_equal(keys, case.keys[idx]), "values do not follow keys"
        eq = f[1:] == f[:-1]
        assert (idx[1:][eq] > idx[:-1][eq]).all(), "not stable"


def run_segmented(args, case, device, barrier, max_over_ranks, world, rank, local):
    """Batched segmented sort (sortSegmentedArray) against a loop of plain
    sortArray calls, one per segment, on the same GPU."""
    import torch
    from mgpu_old_b200 import api

    sorter = GpuSorter(case, device)
    offs_t = torch.from_numpy(case.offsets.astype(np.int32)).to(device)
    engine = api.MgpuSort()
    d = sorter.data
    S = case.num_segments
    stream = torch.cuda.current_stream(device)

    def one_sort():
        api.check(engine.sort_segmented(d, offs_t.data_ptr(), S))

    for _ in range(max(args.warmup, 3)):
        sorter.restore()
        sorter.flush_l2()
        one_sort()
    api.check(engine.synchronize())
    torch.cuda.synchronize()

    engine.enable_kernel_timing(True)
    engine.read_kernel_timing()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    total_ms = 0.0
    for _ in range(args.steps):
        sorter.restore()
        sorter.flush_l2()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_sort()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    barrier()
    clk = clocks.stop()
    kt = engine.read_kernel_timing()
    engine.enable_kernel_timing(False)
    api.check(engine.synchronize())
    keys, vals = sorter.result()
    total_ms = max_over_ranks(total_ms)
    ms_per_step = total_ms / args.steps
    value = case.n * world / (ms_per_step * 1e-3) / 1e6

    # The per-call baseline: every segment in its own 16-byte aligned buffers,
    # one sortArray call each, timed over whole loops.
    sizes = np.diff(case.offsets.astype(np.int64))
    padded = (sizes + 3) // 4 * 4
    poff = np.zeros(S + 1, np.int64)
    np.cumsum(padded, out=poff[1:])
    total = int(poff[-1]) + 2048
    src_k = np.zeros(total, np.uint32)
    src_v = np.zeros(total, np.uint32)
    for i in range(S):
        a, b = int(case.offsets[i]), int(case.offsets[i + 1])
        src_k[poff[i]:poff[i] + (b - a)] = case.keys[a:b]
        src_v[poff[i]:poff[i] + (b - a)] = case.values[0][a:b]
    pk = torch.from_numpy(src_k.view(np.int32)).to(device)
    pv = torch.from_numpy(src_v.view(np.int32)).to(device)
    k0, k1 = pk.clone(), torch.empty_like(pk)
    v0, v1 = pv.clone(), torch.empty_like(pv)
    datas = []
    for i in range(S):
        sd = api.SortData()
        sd.maxElements = sd.numElements = int(sizes[i])
        sd.valueCount = 1
        sd.firstBit, sd.endBit = case.first_bit, case.end_bit
        off = 4 * int(poff[i])
        sd.keys[0], sd.keys[1] = k0.data_ptr() + off, k1.data_ptr() + off
        sd.values[0][0], sd.values[0][1] = v0.data_ptr() + off, v1.data_ptr() + off
        datas.append(sd)
    lib = api.load_library()
    h = engine.handle
    loop_steps = max(1, min(2, args.steps))
    loop_ms = 0.0
    for step in range(loop_steps + 1):
        k0.copy_(pk)
        v0.copy_(pv)
        sorter.flush_l2()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for sd in datas:
            api.check(lib.sortArray(h, ctypes_byref(sd)))
        e1.record(stream)
        e1.synchronize()
        if step > 0:                       # the first loop is a warm-up
            loop_ms += e0.elapsed_time(e1)
    api.check(engine.synchronize())
    loop_ms /= loop_steps
    lk = k0.cpu().numpy().view(np.uint32)
    lv = v0.cpu().numpy().view(np.uint32)
    same = True
    for i in range(S):
        a, b = int(case.offsets[i]), int(case.offsets[i + 1])
        p0 = int(poff[i])
        same &= np.array_equal(keys[a:b], lk[p0:p0 + (b - a)])
        same &= np.array_equal(vals[0][a:b], lv[p0:p0 + (b - a)])
    if not same:
        raise AssertionError("batched result differs from the per-call sortArray loop")

    # End to end through the C ABI with pinned host buffers: every step
    # copies the keys, values and segment offsets in, sorts and copies the
    # keys and values out. As for sortArray, E2E_LANES batches are in flight
    # (one engine, stream, offsets array and set of device buffers each);
    # the one-batch-at-a-time figure is reported beside it.
    pin_k = torch.from_numpy(case.keys.view(np.int32)).pin_memory()
    pin_v = torch.from_numpy(case.values[0].view(np.int32)).pin_memory()
    pin_o = torch.from_numpy(case.offsets.astype(np.int32)).pin_memory()
    lanes = [(sorter, engine, offs_t)] + \
        [(GpuSorter(case, device), api.MgpuSort(), torch.empty_like(offs_t))
         for _ in range(E2E_LANES - 1)]
    lane_streams = [torch.cuda.Stream(device) for _ in lanes]
    outs = [(torch.empty(case.n, dtype=torch.int32).pin_memory(),
             torch.empty(case.n, dtype=torch.int32).pin_memory()) for _ in lanes]

    def e2e_step(j):
        srt, eng, offs = lanes[j]
        st = lane_streams[j]
        dd = srt.data
        out_k, out_v = outs[j]
        with torch.cuda.stream(st):
            srt.bufs[dd.keys[0]][:case.n].copy_(pin_k, non_blocking=True)
            srt.bufs[dd.values[0][0]][:case.n].copy_(pin_v, non_blocking=True)
            offs.copy_(pin_o, non_blocking=True)
            api.check(eng.sort_segmented(dd, offs.data_ptr(), S, st.cuda_stream))
            out_k.copy_(srt.bufs[dd.keys[0]][:case.n], non_blocking=True)
            out_v.copy_(srt.bufs[dd.values[0][0]][:case.n], non_blocking=True)

    def e2e_run(steps, inflight):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(lane_streams[0])
        for st in lane_streams[1:inflight]:
            st.wait_event(e0)
        for j in range(steps):
            if inflight == 1 and j:
                lane_streams[0].synchronize()
            e2e_step(j % inflight)
        for st in lane_streams[1:inflight]:
            done = torch.cuda.Event()
            done.record(st)
            lane_streams[0].wait_event(done)
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(lane_streams[0])
        e1.synchronize()
        return e0.elapsed_time(e1)

    e2e_run(len(lanes), len(lanes))   # warm every engine and the copy paths
    barrier()
    e2e_ms = max_over_ranks(e2e_run(args.steps, len(lanes)))
    serial_steps = max(2, args.steps // 4)
    e2e_serial_ms = max_over_ranks(e2e_run(serial_steps, 1))
    for _, eng, _ in lanes:
        api.check(eng.synchronize())
    last = (args.steps - 1) % len(lanes)
    if not (np.array_equal(outs[last][0].numpy().view(np.uint32), keys)
            and np.array_equal(outs[last][1].numpy().view(np.uint32), vals[0])):
        raise AssertionError("end-to-end result differs from the device-timed run")
    e2e_value = case.n * world / (e2e_ms / args.steps * 1e-3) / 1e6
    e2e_serial = case.n * world / (e2e_serial_ms / serial_steps * 1e-3) / 1e6
    for _, eng, _ in lanes[1:]:
        eng.release()
    del lanes

    peak, peak_src = hbm_peak()
    large = sizes[sizes > 4096].sum()
    passes = len(_plan(case))
    pass_bytes = 2 * int(large) * 4 * 2
    pass_ms = kt["pass_ms"] / max(kt["pass_launches"], 1)
    achieved = pass_bytes / (pass_ms * 1e-3) / 1e9
    alg = workloads.algorithmic_bytes(case.n, case.first_bit, case.end_bit, case.value_count)
    line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded numpy)",
            "config": workload_config(case, args, {"segments": S,
                                                  "large_segment_elements": int(large)}),
            "e2e": {"value": round(e2e_value, 1), "unit": UNIT,
                    "h2d_bytes_per_step": 8 * case.n + 4 * (S + 1),
                    "d2h_bytes_per_step": 8 * case.n, "batches_in_flight": E2E_LANES,
                    "one_batch_at_a_time": round(e2e_serial, 1)},
            "per_call_loop": {"ms_per_step": round(loop_ms, 3),
                              "Mkeys_s": round(case.n / (loop_ms * 1e-3) / 1e6, 1),
                              "speedup": round(loop_ms / ms_per_step, 2),
                              "identical_output": True},
            "gpu_launches": 2 + 2 * kt["upsweep_launches"] + 3 * kt["pass_launches"],
            "roofline": {"bound": "hbm", "kernel": "seg pass (count+scan+sort)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_src,
                         "traffic": None, "bytes_per_launch": pass_bytes,
                         "avg_launch_ms": round(pass_ms, 5),
                         "whole_sort": {"alg_bytes": alg,
                                        "achieved": round(alg / (ms_per_step * 1e-3) / 1e9, 1),
                                        "frac": round(alg / (ms_per_step * 1e-3) / 1e9 / peak, 4)},
                         "small_segments_avg_ms": round(
                             kt["upsweep_ms"] / max(kt["upsweep_launches"], 1), 5)},
            "clocks": clk}
    engine.release()
    return line


def served_requests(count, seed=11):
    """Served workload: sizes log-uniform in [1024, 16777216], half of the
    requests keys-only and half key + one value, endBit uniform in {16, 24,
    32}. Returns (sizes, has_values, end_bits, input offsets)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1024), np.log(16_777_216), count)).astype(np.int64)
    has_values = rng.integers(0, 2, count).astype(bool)
    end_bits = rng.choice([16, 24, 32], count)
    return sizes, has_values, end_bits, rng


def run_served(args, device, local):
    """Served sort requests with Poisson arrivals: the sort server against
    serial plain sortArray (one request at a time: copy in, sortArrayAsync,
    copy out), at offered loads of 0.5x, 0.8x and 1.0x the serial capacity.
    Latency is arrival (submission) to results in host memory."""
    import threading
    import torch
    from mgpu_old_b200 import api

    R = args.requests
    sizes, has_values, end_bits, rng = served_requests(R)
    # Input data: slices of one page-locked pool of random keys and values.
    pool_n = 1 << 25
    keys_pool = torch.from_numpy(rng.integers(0, 1 << 32, pool_n, dtype=np.uint64)
                                 .astype(np.uint32).view(np.int32)).pin_memory()
    vals_pool = torch.arange(pool_n, dtype=torch.int32).pin_memory()
    starts = rng.integers(0, pool_n - sizes + 1)
    # Outputs: a ring in page-locked memory (results are checked in the tests).
    ring_n = 1 << 27
    out_k = torch.empty(ring_n, dtype=torch.int32).pin_memory()
    out_v = torch.empty(ring_n, dtype=torch.int32).pin_memory()
    ring_at = (np.cumsum(sizes) - sizes) % (ring_n - int(sizes.max()))
    total_elems = int(sizes.sum())
    kptr, vptr = keys_pool.data_ptr(), vals_pool.data_ptr()
    okp, ovp = out_k.data_ptr(), out_v.data_ptr()

    # Serial baseline: one engine, one stream, device buffers for the largest
    # request.
    engine = api.MgpuSort()
    nmax = int(sizes.max())
    dk = [torch.empty(nmax, dtype=torch.int32, device=device) for _ in range(2)]
    dv = [torch.empty(nmax, dtype=torch.int32, device=device) for _ in range(2)]
    stream = torch.cuda.Stream(device)

    def serial(arrivals):
        lat = np.zeros(R)
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for i in range(R):
                now = time.perf_counter() - t0
                if arrivals[i] > now:
                    time.sleep(arrivals[i] - now)
                n = int(sizes[i])
                a = int(starts[i])
                dk[0][:n].copy_(keys_pool[a:a + n], non_blocking=True)
                d = api.SortData()
                d.maxElements = d.numElements = n
                d.firstBit, d.endBit = 0, int(end_bits[i])
                d.keys[0], d.keys[1] = dk[0].data_ptr(), dk[1].data_ptr()
                if has_values[i]:
                    dv[0][:n].copy_(vals_pool[a:a + n], non_blocking=True)
                    d.valueCount = 1
                    d.values[0][0], d.values[0][1] = dv[0].data_ptr(), dv[1].data_ptr()
                api.check(engine.sort_array_async(d, stream.cuda_stream))
                o = int(ring_at[i])
                res_k = dk[0] if d.keys[0] == dk[0].data_ptr() else dk[1]
                out_k[o:o + n].copy_(res_k[:n], non_blocking=True)
                if has_values[i]:
                    res_v = dv[0] if d.values[0][0] == dv[0].data_ptr() else dv[1]
                    out_v[o:o + n].copy_(res_v[:n], non_blocking=True)
                stream.synchronize()
                lat[i] = time.perf_counter() - t0 - arrivals[i]
        span = time.perf_counter() - t0
        return lat, span

    def served(arrivals, server):
        tickets = [None] * R
        lat = np.zeros(R)
        t0 = time.perf_counter()

        def waiter():
            for i in range(R):
                while tickets[i] is None:
                    time.sleep(0.0001)
                st, lat[i] = server.wait(tickets[i])
                api.check(st)

        th = threading.Thread(target=waiter)
        th.start()
        for i in range(R):
            now = time.perf_counter() - t0
            if arrivals[i] > now:
                time.sleep(arrivals[i] - now)
            n = int(sizes[i])
            a = 4 * int(starts[i])
            o = 4 * int(ring_at[i])
            tickets[i] = server.submit(kptr + a, vptr + a if has_values[i] else None, n, 0,
                                       int(end_bits[i]), okp + o,
                                       ovp + o if has_values[i] else None)
        th.join()
        span = time.perf_counter() - t0
        return lat, span

    # Capacity of the serial path: all requests present at t = 0.
    serial(np.zeros(R))                       # warm-up
    lat0, span0 = serial(np.zeros(R))
    capacity = R / span0                      # requests per second
    server = api.SortServer(memory_budget=args.server_budget << 30, slots=args.server_slots,
                            coalesce_max=1 << 20)
    served(np.zeros(R), server)               # warm-up: grows the memory pool
    results = []
    for load in (0.5, 0.8, 1.0):
        rate = load * capacity
        arrivals = np.cumsum(rng.exponential(1.0 / rate, R))
        sl, sspan = serial(arrivals)
        vl, vspan = served(arrivals, server)
        results.append({"offered_load": load, "rate_rps": round(rate, 1),
                        "server": {"Mkeys_s": round(total_elems / vspan / 1e6, 1),
                                   "p50_ms": round(float(np.percentile(vl, 50)) * 1e3, 3),
                                   "p99_ms": round(float(np.percentile(vl, 99)) * 1e3, 3)},
                        "serial_sortArray": {"Mkeys_s": round(total_elems / sspan / 1e6, 1),
                                             "p50_ms": round(float(np.percentile(sl, 50)) * 1e3, 3),
                                             "p99_ms": round(float(np.percentile(sl, 99)) * 1e3, 3)}})
    # Saturation: everything at t = 0. This is the headline value; the clocks
    # are sampled over it.
    clocks = ClockSampler(local)
    clocks.start()
    vl, vspan = served(np.zeros(R), server)
    clk = clocks.stop()
    server.close()
    engine.release()
    best = total_elems / vspan / 1e6
    line = {"metric": METRIC, "value": round(best, 1), "unit": UNIT, "n_gpus": 1,
            "steps": R, "warmup": args.warmup, "ms_per_step": round(vspan / R * 1e3, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded numpy)",
            "config": {"workload": "served_requests", "requests": R,
                       "sizes": "log-uniform [1024, 16777216]",
                       "mix": "50% keys-only / 50% key+value, endBit in {16, 24, 32}",
                       "arrivals": "Poisson at 0.5/0.8/1.0 x serial capacity",
                       "memory_budget_GiB": args.server_budget, "slots": args.server_slots,
                       "elements": total_elems, "parallelism": "replicas1"},
            "e2e": {"value": round(best, 1), "unit": UNIT,
                    "h2d_bytes_per_step": int(4 * (sizes + sizes * has_values).sum() / R),
                    "d2h_bytes_per_step": int(4 * (sizes + sizes * has_values).sum() / R)},
            "serial_capacity": {"requests_per_s": round(capacity, 1),
                                "Mkeys_s": round(total_elems / span0 / 1e6, 1)},
            "saturated_server": {"Mkeys_s": round(best, 1),
                                 "p50_ms": round(float(np.percentile(vl, 50)) * 1e3, 3),
                                 "p99_ms": round(float(np.percentile(vl, 99)) * 1e3, 3)},
            "loads": results, "clocks": clk}
    return line


def ctypes_byref(x):
    import ctypes
    return ctypes.byref(x)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from mgpu_old_b200 import replicas
    reps = replicas.from_env("nccl")
    world, rank, local, device = reps.world, reps.rank, reps.local, reps.device
    barrier, max_over_ranks = reps.barrier, reps.max_over_ranks

    from mgpu_old_b200 import api
    api.load_library()
    if args.workload == "served":
        line = run_served(args, device, local)
        reps.close()
        if rank == 0:
            print(json.dumps(line))
        return 0
    if args.workload == "bwt":
        line = run_bwt(args, barrier, max_over_ranks, world, rank, local)
        reps.close()
        if rank == 0:
            print(json.dumps(line))
        return 0
    case = workloads.WORKLOADS[args.workload]()
    if isinstance(case, workloads.SegmentedCase):
        line = run_segmented(args, case, device, barrier, max_over_ranks, world, rank, local)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_segmented(case)
        reps.close()
        if rank == 0:
            print(json.dumps(line))
        return 0
    sorter = GpuSorter(case, device)
    engine = api.MgpuSort()
    d = sorter.data
    stream = torch.cuda.current_stream(device)

    def one_sort():
        if case.key_type:
            api.check(engine.sort_array_typed(d, case.key_type, stream.cuda_stream))
        else:
            api.check(engine.sort_array(d))

    # Warm-up.
    for _ in range(max(args.warmup, 3)):
        sorter.restore()
        sorter.flush_l2()
        one_sort()
    api.check(engine.synchronize())
    torch.cuda.synchronize()
    keys, vals = sorter.result()
    verify(case, keys, vals)

    if args.profile_only:
        for _ in range(args.steps):
            sorter.restore()
            sorter.flush_l2()
            one_sort()
        api.check(engine.synchronize())
        torch.cuda.synchronize()
        engine.release()
        return 0

    # Timed device-resident steps: CUDA events around each sort on its
    # stream, inputs restored and L2 flushed before each step (outside the
    # events).
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()

    def timed_steps():
        total = 0.0
        for _ in range(args.steps):
            sorter.restore()
            sorter.flush_l2()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            one_sort()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total

    total_ms = timed_steps()
    torch.cuda.synchronize()
    barrier()
    # The same steps again with an event pair around every kernel launch of
    # the engine: per-launch durations for the roofline. (The events between
    # launches cost a few percent of the step time, so `value` comes from
    # the run without them.)
    engine.enable_kernel_timing(True)
    engine.read_kernel_timing()
    timed_ms = timed_steps()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    kt = engine.read_kernel_timing()
    engine.enable_kernel_timing(False)
    api.check(engine.synchronize())
    keys, vals = sorter.result()
    verify(case, keys, vals)

    total_ms = max_over_ranks(total_ms)
    ms_per_step = total_ms / args.steps
    value = case.n * world / (ms_per_step * 1e-3) / 1e6

    # End to end through the C ABI with pinned host buffers: every step
    # copies its inputs in, sorts (sortArrayAsync) and copies the sorted keys
    # and values out. E2E_LANES batches are in flight, each with its own
    # engine, stream and device buffers, as a caller streaming batches
    # through the library would run it: one batch's copies in overlap
    # another's copies out, and with three lanes a batch's copy in never
    # waits for the copy out of the batch before it on the same lane. CUDA
    # events on the streams bracket all steps.
    extra = [(GpuSorter(case, device), api.MgpuSort()) for _ in range(E2E_LANES - 1)]
    lanes = [(sorter, engine, torch.cuda.Stream(device))] + \
        [(srt, eng, torch.cuda.Stream(device)) for srt, eng in extra]
    pinned_in = [torch.from_numpy(case.keys.view(np.int32)).pin_memory()] + \
        [torch.from_numpy(v.view(np.int32)).pin_memory() for v in case.values]
    pinned_out = [[torch.empty(case.n, dtype=torch.int32).pin_memory()
                   for _ in range(1 + sorter.arrays)] for _ in lanes]
    h2d = 4 * case.n * len(pinned_in)
    d2h = 4 * case.n * len(pinned_out[0])

    def e2e_step(j):
        srt, eng, st = lanes[j % len(lanes)]
        dd = srt.data
        out = pinned_out[j % len(lanes)]
        with torch.cuda.stream(st):
            srt.bufs[dd.keys[0]][:case.n].copy_(pinned_in[0], non_blocking=True)
            for i in range(len(case.values)):
                srt.bufs[dd.values[i][0]][:case.n].copy_(pinned_in[1 + i], non_blocking=True)
            if case.key_type:
                api.check(eng.sort_array_typed(dd, case.key_type, st.cuda_stream))
            else:
                api.check(eng.sort_array_async(dd, st.cuda_stream))
            out[0].copy_(srt.bufs[dd.keys[0]][:case.n], non_blocking=True)
            for i in range(srt.arrays):
                out[1 + i].copy_(srt.bufs[dd.values[i][0]][:case.n], non_blocking=True)

    def e2e_run(steps, inflight):
        """Steps spread over the first `inflight` lanes (1: one batch at a
        time, each step waiting for the previous one)."""
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(lanes[0][2])
        for _, _, st in lanes[1:inflight]:
            st.wait_event(e0)
        for j in range(steps):
            if inflight == 1 and j:
                lanes[0][2].synchronize()
            e2e_step(j % inflight)
        for _, _, st in lanes[1:inflight]:
            done = torch.cuda.Event()
            done.record(st)
            lanes[0][2].wait_event(done)
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(lanes[0][2])
        e1.synchronize()
        return e0.elapsed_time(e1)

    e2e_run(len(lanes), len(lanes))   # warm every engine and the copy paths
    barrier()
    e2e_ms = max_over_ranks(e2e_run(args.steps, len(lanes)))
    e2e_serial_ms = max_over_ranks(e2e_run(max(2, args.steps // 4), 1))
    for _, eng, _ in lanes:
        api.check(eng.synchronize())
    last = (args.steps - 1) % len(lanes)
    verify(case, pinned_out[last][0].numpy().view(np.uint32),
           [p.numpy().view(np.uint32) for p in pinned_out[last][1:]])
    e2e_value = case.n * world / (e2e_ms / args.steps * 1e-3) / 1e6
    e2e_serial = case.n * world / (e2e_serial_ms / max(2, args.steps // 4) * 1e-3) / 1e6

    # The copies alone: one step's inputs in on one stream while another
    # step's results go out on a second, no sort. Its rate bounds e2e.
    def copies_only(reps=3):
        (srt_a, _, _), (srt_b, _, _) = lanes[0], lanes[1]
        sa, sb = torch.cuda.Stream(device), torch.cuda.Stream(device)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record()
        sa.wait_event(e0)
        sb.wait_event(e0)
        da, db = srt_a.data, srt_b.data
        for _ in range(reps):
            with torch.cuda.stream(sa):
                srt_a.bufs[da.keys[0]][:case.n].copy_(pinned_in[0], non_blocking=True)
                for i in range(len(case.values)):
                    srt_a.bufs[da.values[i][0]][:case.n].copy_(pinned_in[1 + i],
                                                               non_blocking=True)
            with torch.cuda.stream(sb):
                pinned_out[1][0].copy_(srt_b.bufs[db.keys[0]][:case.n], non_blocking=True)
                for i in range(srt_b.arrays):
                    pinned_out[1][1 + i].copy_(srt_b.bufs[db.values[i][0]][:case.n],
                                               non_blocking=True)
        cur = torch.cuda.current_stream(device)
        for st in (sa, sb):
            ev = torch.cuda.Event()
            ev.record(st)
            cur.wait_event(ev)
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    copy_ms = max_over_ranks(copies_only())
    copy_bound = case.n * world / (copy_ms * 1e-3) / 1e6
    for _, eng in extra:
        eng.release()
    del extra

    # Roofline of the sort kernel of a pass.
    peak, peak_src = hbm_peak()
    arrays = sorter.arrays
    pass_bytes = 2 * case.n * 4 * (1 + arrays)
    pass_launches = max(kt["pass_launches"], 1)
    pass_ms = kt["pass_ms"] / pass_launches
    alg_bytes = workloads.algorithmic_bytes(case.n, case.first_bit, case.end_bit,
                                            case.value_count)
    onesweep = os.environ.get("MGPU_SORT_PASS", "range") == "onesweep"
    kernel = "onesweep_kernel" if onesweep else "sort_kernel"
    # Mid-size and small arrays run the whole sort in one launch (the
    # cooperative sort, or one CTA in shared memory): no count/scan launches
    # and one timed launch per sort, whose algorithmic bytes are the whole
    # sort's.
    if kt["upsweep_launches"] == 0 and kt["pass_launches"] == args.steps:
        kernel = "coop_sort_kernel" if case.n > 4096 else "small_array_kernel"
        pass_bytes = alg_bytes
    achieved = pass_bytes / (pass_ms * 1e-3) / 1e9
    traffic = _ncu_traffic(case.name)
    roofline = {"bound": "hbm", "kernel": kernel,
                "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": peak_src,
                "traffic": traffic,
                "bytes_per_launch": pass_bytes, "avg_launch_ms": round(pass_ms, 5),
                "whole_sort": {"alg_bytes": alg_bytes,
                               "achieved": round(alg_bytes / (ms_per_step * 1e-3) / 1e9, 1),
                               "frac": round(alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak, 4)},
                ("upsweep_avg_ms" if onesweep else "count_scan_avg_ms"):
                    round(kt["upsweep_ms"] / max(kt["upsweep_launches"], 1), 5),
                "kernel_timing": "per-launch events in a second run of the same timed steps "
                                 f"({timed_ms / args.steps:.4f} ms per step with the events)"}

    line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded numpy MT19937)",
            "config": workload_config(case, args),
            "e2e": {"value": round(e2e_value, 1), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "batches_in_flight": E2E_LANES,
                    "one_batch_at_a_time": round(e2e_serial, 1),
                    "copy_bound": {"value": round(copy_bound, 1), "unit": UNIT,
                                   "ms_per_step": round(copy_ms, 4),
                                   "frac": round(e2e_value / copy_bound, 4),
                                   "what": "the step's H2D and D2H copies alone, both "
                                           "directions at once, no sort"}},
            # onesweep: one upsweep per sort and one kernel per pass; range
            # partition: count + scan kernels (one timed entry) and the sort
            # kernel per pass
            "gpu_launches": (1 if onesweep else 2) * kt["upsweep_launches"]
                            + kt["pass_launches"],
            "pass_method": "onesweep" if onesweep else "range",
            "roofline": roofline,
            "clocks": clk}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(case, keys, vals)
    engine.release()
    reps.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


def _ncu_traffic(workload):
    """DRAM bytes per pass launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload)
    except Exception:
        return None


if __name__ == "__main__":
    sys.exit(main())

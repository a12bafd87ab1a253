"""The multi-GPU path of the benchmarks is N independent replicas; its only
collectives are a barrier and the maximum of the ranks' timings. These CPU
tests run that plumbing (mgpu_old_b200/replicas.py) as two gloo ranks, and
the reference arm of bench.py as a non-leader rank."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
from mgpu_old_b200 import replicas
r = replicas.from_env("gloo", timeout_s=60)
# Each rank "timed" a different duration; the job figure uses the slowest.
ms = 10.0 + 5.0 * r.rank
r.barrier()
worst = r.max_over_ranks(ms)
rate = replicas.whole_job_rate(1000, r.world, worst, 1)
r.close()
print(json.dumps({"rank": r.rank, "leader": r.leader, "worst": worst, "rate": rate}))
"""


def run_ranks(world: int):
    port = free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    return outs


def test_two_gloo_ranks_take_the_slowest_timing():
    outs = run_ranks(2)
    assert [o["rank"] for o in outs] == [0, 1]
    assert [o["leader"] for o in outs] == [True, False]
    for o in outs:
        assert o["worst"] == 15.0
        # Two replicas of 1000 units in the slowest rank's 15 ms.
        assert o["rate"] == pytest.approx(2000 / 0.015)


def test_single_rank_needs_no_process_group():
    from mgpu_old_b200 import replicas
    r = replicas.Replicas(1, 0, 0)
    r.barrier()
    assert r.max_over_ranks(3.5) == 3.5
    r.close()


def test_reference_arm_non_leader_rank_exits_quietly():
    """Under torchrun only rank 0 runs and prints the reference arm."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_json_line():
    """The reference arm's JSON line on this host (rank 0, N=1)."""
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "sort Mkeys/s" and line["unit"] == "Mkeys/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] in ("port", "reference")
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"] == "pairs_u32_64M"
    assert line["config"]["n"] == 67_108_864       # the whole workload, no sample
    assert line["steps_timed"] == 1


@pytest.mark.parametrize("workload", ["keys_u32_1M", "pairs_and24_32M"])
def test_reference_arm_never_loads_the_library(workload):
    """The CPU arm runs the reference's CPU path only: after it, the process
    has not mapped libmgpusort_b200.so."""
    code = (
        "import runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',"
        f" '--workload', '{workload}']\n"
        "try:\n"
        f"    runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED' if 'libmgpusort_b200' in maps else 'NOT_LOADED')\n")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr
    out = p.stdout.strip().splitlines()
    line = json.loads(out[-2])
    assert line["impl"] == "reference" and line["config"]["workload"] == workload
    have_ref = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_cpusort.so"))
    expect_kind = "reference" if workload == "keys_u32_1M" and have_ref else "port"
    assert line["cpu_baseline"]["kind"] == expect_kind
    assert out[-1] == "NOT_LOADED"


@pytest.mark.parametrize("workload,metric,unit", [
    ("segments_10k", "sort Mkeys/s", "Mkeys/s"),
    ("multi6_17bit_16M", "sort Mkeys/s", "Mkeys/s"),
    ("served", "sort Mkeys/s", "Mkeys/s"),
    ("bwt", "bwtSortBlock MB/s", "MB/s"),
])
def test_reference_arm_other_workloads(workload, metric, unit):
    """Every workload's reference arm prints one contract line (CPU only)
    and never maps the library."""
    code = (
        "import runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',"
        f" '--workload', '{workload}']\n"
        "try:\n"
        f"    runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED' if 'libmgpusort_b200' in maps else 'NOT_LOADED')\n")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr
    out = p.stdout.strip().splitlines()
    assert out[-1] == "NOT_LOADED"
    line = json.loads(out[-2])
    assert line["impl"] == "reference"
    assert line["metric"] == metric and line["unit"] == unit
    assert line["value"] > 0 and line["higher_is_better"] is True
    for key in ("n_gpus", "steps", "warmup", "ms_per_step", "scaling", "vs_baseline", "dtype",
                "data", "config"):
        assert key in line, key
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert cb["value"] == line["value"] and cb["unit"] == unit and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": unit, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}

"""The multi-GPU path of the benchmark is replicas (every rank renders its own frame; no data-path
collective): its process-group plumbing on CPU with gloo, world size 2 — the max of the step
times over ranks, the barriers, and the reference arm, which only rank 0 runs."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import bench
world, rank, _ = bench.dist_init("gloo")
bench.barrier(world)
m = bench.max_over_ranks(world, 10.0 + rank)
bench.barrier(world)
print(json.dumps({{"rank": rank, "world": world, "max": m}}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(code: str, world: int, extra_env=None, timeout=120):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, e[-2000:]
        outs.append(o)
    return outs


def test_max_over_ranks_and_barrier_with_gloo():
    import json

    outs = _launch(WORKER.format(root=ROOT), 2)
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 11.0 for r in res)


def test_reference_arm_runs_on_rank_zero_only():
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); import bench, argparse; "
            "a = argparse.Namespace(workload='room_256_4k', steps=1, warmup=0); "
            "import os; r = int(os.environ['RANK']); "
            "rc = bench.run_reference(a) if r == 1 else 0; print('rc', rc)")
    outs = _launch(code, 2)
    assert outs[1].strip().splitlines()[-1] == "rc 0"  # rank 1 returns at once, without work


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` needs no GPU: on a small workload it prints one JSON line with
    the benchmark's metric, a cpu_baseline describing the run and an e2e with no copies."""
    import json

    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "room_256_4k", "--steps", "2", "--warmup", "1"], env=env, capture_output=True, text=True,
                       timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [s for s in r.stdout.splitlines() if s.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    import bench

    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["ms_per_step"] == line["value"] and line["higher_is_better"] is False
    assert line["steps"] == 2 and line["warmup"] == 1 and line["n_gpus"] == 1
    b = line["cpu_baseline"]
    assert b["value"] == line["value"] and b["kind"] in ("port", "reference") and b["cores"] >= 1 and b["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "room_256_4k"
    # what the gather got from the host, per step
    assert len(b["per_step_values"]) == 2 and len(b["per_step_cpu_seconds_per_second"]) == 2
    assert 0 < b["cpu_seconds_per_second"] <= b["cores"] + 1
    assert set(b["context_switches"]) == {"involuntary", "voluntary"}
    if b["host_cpu"] is not None:
        assert 0 <= b["host_cpu"]["busy"] <= 1 and 0 <= b["host_cpu"]["steal"] <= 1


def test_host_cpu_readers():
    """The host and cgroup CPU readers the baseline records: well-formed on this machine, whatever
    its cgroup version."""
    import bench

    h = bench.host_cpu_times()
    if h is not None:
        busy, steal, total = h
        assert 0 <= busy <= total and 0 <= steal <= total
    cg = bench.cgroup_cpu()
    assert set(cg) == {"quota_cores", "throttled_s", "nr_throttled"}
    assert cg["quota_cores"] is None or cg["quota_cores"] > 0
    assert cg["throttled_s"] is None or cg["throttled_s"] >= 0
    assert bench.host_threads() >= 1


def test_reference_arm_loads_no_gpu_library():
    """The reference arm makes its inputs with the scene generator built alone (oracle/libinputs.so)
    and times the oracle's CPU gather: the process maps neither libarc.so nor any CUDA library."""
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); import bench, argparse; "
            "a = argparse.Namespace(workload='room_256_4k', steps=1, warmup=0); bench.run_reference(a); "
            "maps = open('/proc/self/maps').read(); "
            "print('LIBS', sorted({l.split()[-1] for l in maps.splitlines() if '.so' in l}))")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    libs = [s for s in r.stdout.splitlines() if s.startswith("LIBS")][0]
    assert "liboracle.so" in libs and "libinputs.so" in libs
    assert "libarc.so" not in libs and "libcuda" not in libs and "libcudart" not in libs and "libtorch" not in libs

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

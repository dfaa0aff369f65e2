"""The multi-GPU form of bench.py: independent replicas, one process per GPU.

Host-side logic only, on CPU with two gloo ranks: the job time is the slowest
rank's time (an all-reduce MAX, the same collective the GPU run issues over
NCCL), the value counts every rank's products, and the reference arm does its
work on rank 0 alone.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import torch
import torch.distributed as dist
import bench

rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:" + os.environ["MASTER_PORT"], rank=rank,
                        world_size=world)

def reduce_max(v):
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()

dist.barrier()
ms, us = bench.job_time(10.0 + 2.5 * rank, 40, world, reduce_max)
dist.barrier()
print(json.dumps({"rank": rank, "ms": ms, "us": us}))
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replica_job_time_is_max_over_ranks_and_counts_all_products(tmp_path):
    world = 2
    port = str(free_port())
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["ms"] == pytest.approx(12.5)                      # the slower rank's time
        assert o["us"] == pytest.approx(12.5e3 / (40 * world))     # every rank's products


def test_job_time_single_process():
    import bench
    ms, us = bench.job_time(8.0, 100, 1, reduce_max=None)
    assert (ms, us) == (8.0, 80.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("Args", (), {"workload": "N4096_W256", "steps": 1, "warmup": 0, "gpus": 2})()
    bench.run_reference(args)
    assert capsys.readouterr().out == ""

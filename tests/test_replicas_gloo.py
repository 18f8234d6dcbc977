"""Multi-process plumbing of `bench.py --gpus N` (replicas, one process per
GPU) on CPU with the gloo backend, world size 2: timing is the max over
ranks, and the reference arm runs on rank 0 only."""

import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


WORKER = r"""
import os, sys, datetime
sys.path.insert(0, {repo!r})
import torch.distributed as dist
import bench
dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
r = dist.get_rank()
v = bench.max_over_ranks(10.0 + 5.0 * r, dist)
assert v == 15.0, v
v = bench.max_over_ranks(-1.0 - r, dist)
assert v == -1.0, v
dist.barrier()
dist.destroy_process_group()
print("ok", r)
"""


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE="2", LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(repo=REPO)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
    assert sorted(o.strip() for o, _ in outs) == ["ok 0", "ok 1"]


def test_max_over_ranks_without_group():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""

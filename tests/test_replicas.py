"""The multi-GPU path of bench.py on the CPU: replicas (one job per rank, no
data-path collective) combined by the max of the ranks' times over a gloo
process group of two ranks, and the reference arm running on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
rank = int(os.environ["RANK"])
dist.init_process_group("gloo")
slowest = bench.reduce_max_over_ranks(1.5 + rank, dist, "cpu")   # rank 1 is the slow one
value = bench.replica_throughput(int(os.environ["WORLD_SIZE"]), 1000, 4, slowest)
# the reference arm: rank 0 alone does work; other ranks return at once
class A: pass
a = A(); a.gpus = 2; a.steps = 1; a.warmup = 0
if rank != 0:
    bench.run_reference_arm(a, None)  # would fail on a None workload if it did any work
print(json.dumps({{"rank": rank, "slowest": slowest, "value": value}}), flush=True)
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_combine_by_the_slowest():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    try:
        for p in procs:
            out, err = p.communicate(timeout=120)
            assert p.returncode == 0, err
            outs.append(out.strip().splitlines()[-1])
    finally:
        for p in procs:  # the exact processes started here
            if p.poll() is None:
                p.kill()
                p.wait()
    import json

    res = [json.loads(o) for o in outs]
    for r in res:
        assert r["slowest"] == pytest.approx(2.5)           # max over ranks, seen by both
        assert r["value"] == pytest.approx(2 * 1000 * 4 / 2.5)  # whole-job reads/s of both replicas

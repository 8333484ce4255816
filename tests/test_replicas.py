"""The multi-GPU path of bench.py is replicas only: every rank runs its own
copy of the workload, and the process group carries nothing but the timing
reductions (whole-job throughput = units of all ranks / slowest rank's time)
and the reference arm's rank-0 rule.  World size 2 on CPU with gloo."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, os, sys
sys.path.insert(0, %r)
import bench
world, rank, local = bench.dist_setup("gloo")
units = 1000.0 * (rank + 1)          # rank 0: 1000 units, rank 1: 2000
ms = 10.0 * (rank + 1)               # rank 1 is the slowest: 20 ms
value = bench.replica_value(units, ms, world)
mx = bench.dist_max(ms, world)
sm = bench.dist_sum(units, world)
bench.barrier(world)

class A:
    ref_steps = 1; gpus = world; steps = 1; warmup = 0
printed = []
orig = bench.reference_sample
bench.reference_sample = lambda w, steps: dict(value=123.0, seconds=1.0, markers=7, procs=2,
                                               per_process=61.5, sample="stub")
import io, contextlib
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    bench.run_reference_arm(A(), dict(name="w", n=(8, 8, 8)), world, rank)
print(json.dumps(dict(rank=rank, value=value, max=mx, sum=sm, ref=buf.getvalue())))
import torch.distributed as dist
dist.destroy_process_group()
''' % ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replica_reductions_over_two_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err.decode()[-2000:]
        outs.append(json.loads(out.decode().strip().splitlines()[-1]))
    for o in outs:
        assert o["max"] == 20.0 and o["sum"] == 3000.0
        assert o["value"] == pytest.approx(3000.0 / 0.020)
    # The reference arm prints one line, on rank 0 only.
    by_rank = {o["rank"]: o for o in outs}
    assert by_rank[1]["ref"] == ""
    line = json.loads(by_rank[0]["ref"])
    assert line["impl"] == "reference" and line["value"] == 123.0

"""The bench's multi-rank plumbing on CPU: two ranks over gloo, one process
each, started the way torchrun starts the bench (RANK / WORLD_SIZE /
MASTER_ADDR=127.0.0.1 in the environment).  Every rank passes the barrier,
the job's time is the slowest rank's (max over ranks), and the reference arm
runs on rank 0 alone -- rank 1 returns at once without touching the oracle."""
import json
import os
import socket
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import datetime, json, os, sys, time
sys.path.insert(0, os.environ["REPO"])
import torch.distributed as dist
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
bench.barrier(world)
slowest = bench.max_over_ranks(10.0 * (rank + 1), world)
t0 = time.perf_counter()
skipped = bench.run_reference(None) if rank == 1 else None   # rank != 0: returns before any work
ref_s = time.perf_counter() - t0
bench.barrier(world)
dist.destroy_process_group()
print(json.dumps({"rank": rank, "slowest": slowest, "skipped": skipped, "ref_s": ref_s}))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_barrier_max_and_reference_rank0_only():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, REPO=REPO, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    assert [d["slowest"] for d in outs] == [20.0, 20.0]
    assert outs[1]["skipped"] is None and outs[1]["ref_s"] < 1.0

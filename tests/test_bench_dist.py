"""The multi-rank path of bench.py on the CPU: two gloo ranks (127.0.0.1)
exercise the process-group set-up, the disjoint per-rank event seeds (weak
scaling, no data-path collective), the max-over-ranks timing and the
reference arm's rank-0-only rule.  No GPU is touched."""
import json
import os
import socket
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
import torch.distributed as dist
bench.init_dist("gloo", timeout_s=60)
rank, world, _ = bench.dist_env()
seeds = bench.event_seeds(rank, 64)
allseeds = [None] * world
dist.all_gather_object(allseeds, seeds)
bench.barrier()
slowest = bench.max_over_ranks(1.5 + rank)
class A: steps = 3; warmup = 3
if rank != 0:
    bench.reference_arm(A())  # returns at once on ranks other than 0
bench.barrier()
print(json.dumps({"rank": rank, "world": world, "slowest": slowest,
                  "overlap": len(set(allseeds[0]) & set(allseeds[1])), "n": [len(x) for x in allseeds]}))
dist.destroy_process_group()
"""


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, REPO], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for rank, p in enumerate(procs):
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        lines = out.strip().splitlines()
        if rank == 1:
            assert len(lines) == 1  # the reference arm printed nothing there
        outs.append(json.loads(lines[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["slowest"] == 2.5          # the max over ranks, seen by every rank
        assert o["overlap"] == 0 and o["n"] == [64, 64]
    assert {o["rank"] for o in outs} == {0, 1}

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


ENSEMBLE_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/softx-d-21-00092_b200")
import bench
import torch.distributed as dist
from jimwlk.dist import allreduce_ensemble
bench.init_dist("gloo", timeout_s=60)
rank, world, _ = bench.dist_env()
rng = np.random.default_rng(100 + rank)
s = rng.standard_normal((16, 16)) + 0j
e = s.real ** 2 + 0j
parts = [None] * world
dist.all_gather_object(parts, (s.copy(), e.copy()))
allreduce_ensemble(s, e)
want_s = sum(p[0] for p in parts)
want_e = sum(p[1] for p in parts)
print(json.dumps({"rank": rank, "ds": float(np.abs(s - want_s).max()), "de": float(np.abs(e - want_e).max()),
                  "imag": float(np.abs(s.imag).max())}))
dist.destroy_process_group()
"""


def test_ensemble_allreduce_over_two_gloo_ranks():
    """The ensemble of two ranks' events is the sum of their ensemble fields,
    as every rank sees it after allreduce_ensemble."""
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", ENSEMBLE_CHILD, REPO], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        o = json.loads(out.strip().splitlines()[-1])
        assert o["ds"] < 1e-14 and o["de"] < 1e-14 and o["imag"] == 0.0

"""bench.py's multi-rank arithmetic on CPU: world_size-2 gloo ranks.  Each
replica times its own device; the job's step time is the slowest rank's
(an all-reduce MAX that every rank joins), and the job's value counts every
rank's rays over that time."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

RANK_CODE = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["BENCH_ROOT"])
import torch.distributed as dist
import bench
rank, world, _ = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
mine = [0.50, 0.75][rank]
ms = bench.max_over_ranks(mine, world, "cpu")
dist.barrier()
print(json.dumps({"rank": rank, "ms": ms, "value": bench.job_value(world, 2_000_000, ms)}), flush=True)
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_slowest_rank():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   LOCAL_RANK=str(rank), BENCH_ROOT=str(ROOT))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_CODE], env=env, cwd=ROOT, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    want = 2 * 2_000_000 / (0.75e-3) / 1e9
    for o in outs:
        assert o["ms"] == 0.75
        assert abs(o["value"] - want) < 1e-12 * want


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(0.4, 1, "cpu") == 0.4
    assert bench.job_value(1, 1_000_000, 0.5) == 1_000_000 / 0.5e-3 / 1e9

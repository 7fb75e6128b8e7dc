"""Replicas plumbing of bench.py on CPU (gloo, world size 2): the process
group, the max over ranks of the per-rank device times, the weak-scaling
value, scene sharding, and the reference arm doing no work off rank 0.  The
GPU work of each rank is independent (no data-path collective), so this is
the whole multi-process path."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

RANK_CODE = r"""
import json, os, sys
sys.path.insert(0, os.getcwd())
import bench
rank, _, world = bench.dist_env()
assert bench.dist_init("gloo", timeout_s=60)
ms = 100.0 + 50.0 * rank          # this rank's device time
worst = bench.max_over_ranks(ms, "cpu")
mine = bench.shard(list(range(7)), rank, world)
value = bench.weak_value(1, world, 10, worst)
bench.run_reference(None) if rank != 0 else None   # returns at once off rank 0
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({"rank": rank, "world": world, "worst": worst, "mine": mine, "value": value}))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_CODE], cwd=ROOT, env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    out = []
    for p in procs:
        so, se = p.communicate(timeout=180)
        assert p.returncode == 0, se[-2000:]
        out.append(json.loads(so.strip().splitlines()[-1]))
    out.sort(key=lambda d: d["rank"])
    for d in out:
        assert d["world"] == 2
        assert d["worst"] == 150.0                 # the slower rank's time on every rank
        assert abs(d["value"] - 2 * 10 / 0.150) < 1e-9
    assert out[0]["mine"] == [0, 2, 4, 6] and out[1]["mine"] == [1, 3, 5]


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench

    env = {k: os.environ.get(k) for k in ("RANK", "WORLD_SIZE")}
    try:
        os.environ.pop("RANK", None)
        os.environ.pop("WORLD_SIZE", None)
        assert bench.dist_init("gloo") is False
        assert bench.max_over_ranks(12.5, "cpu") == 12.5
        assert bench.shard([1, 2, 3], 0, 1) == [1, 2, 3]
    finally:
        for k, v in env.items():
            if v is not None:
                os.environ[k] = v

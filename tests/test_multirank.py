"""Multi-rank bench logic on CPU (gloo, world size 2): max-over-ranks timing,
whole-job aggregation, and the reference arm's rank-0-only rule."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = [10.0, 25.0][rank]
    t = bench.max_over_ranks(local, world, torch.device("cpu"))
    out[rank] = (t, bench.aggregate_rate(world, 1000, 4, t))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 25.0
    assert abs(res[0][1] - 2 * 1000 * 3 * 4 / 0.025) < 1e-6


def test_reference_arm_non_zero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""

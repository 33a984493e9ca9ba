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


def _shard_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from dgsem_b200 import sharding
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = bench.batched_meshes()
    mine = [i for i, _ in sharding.local_meshes(specs, rank, world)]
    cost = sum(sharding.mesh_cost(specs[i][0], specs[i][1]) for i in mine)
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, cost))
    out[rank] = gathered
    dist.barrier()
    dist.destroy_process_group()


def test_batched_meshes_sharded_over_ranks_gloo_world2():
    """Every rank computes the same placement without communication: the
    256 meshes of the batched workload are covered exactly once and the two
    ranks' loads are within the largest mesh's cost of each other."""
    sys.path.insert(0, ROOT)
    import bench
    from dgsem_b200 import sharding
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_shard_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    (a, ca), (b, cb) = res[0]
    assert sorted(a + b) == list(range(256)) and not set(a) & set(b)
    specs = bench.batched_meshes()
    biggest = max(sharding.mesh_cost(s[0], s[1]) for s in specs)
    assert abs(ca - cb) <= biggest


def test_assign_meshes_lpt_properties():
    from dgsem_b200 import sharding
    costs = [7.0, 5.0, 4.0, 4.0, 3.0, 3.0, 3.0, 1.0]
    parts = sharding.assign_meshes(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= 4.0 / 3.0 * (sum(costs) / 3) + max(costs)  # LPT bound
    assert sharding.assign_meshes(costs, 1) == [list(range(len(costs)))]

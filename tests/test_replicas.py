"""Replica (multi-GPU) rank logic on CPU with world_size 2 over gloo."""
import os
import socket

import pytest
import torch.multiprocessing as tmp

from lgcr import replicas as R


def test_shard_is_disjoint_and_covering():
    items = list(range(32))
    parts = [R.shard(items, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == items
    assert not set(parts[0]) & set(parts[1])
    assert len({R.frame_seed(1000, r, i) for r in range(4) for i in range(32)}) == 128


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = R.max_over_ranks(10.0 + rank)
    items = R.shard(list(range(10)), rank, world)
    total = [0.0]
    import torch
    t = torch.tensor([float(len(items))])
    dist.all_reduce(t)
    out[rank] = (got, float(t.item()))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_max_over_ranks_gloo_world2():
    world = 2
    manager = tmp.Manager()
    out = manager.dict()
    tmp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        assert out[r][0] == 11.0             # max over ranks
        assert out[r][1] == 10.0             # shards cover all frames
    assert R.aggregate_throughput([100, 100], 2.0) == 100.0


def test_relaunch_starts_one_process_per_replica(capfd):
    import json
    child = os.path.join(os.path.dirname(os.path.abspath(__file__)), "replica_child.py")
    assert R.launch_command(child, ["--x"], 2, 1234)[-2:] == [child, "--x"]
    rc = R.relaunch(child, [], 2, timeout_s=300)
    assert rc == 0
    line = [l for l in capfd.readouterr().out.splitlines() if l.startswith("{")][-1]
    assert json.loads(line) == {"world": 2, "max": 11.0, "frames": 32.0}

"""Multi-GPU form of the Recon path: independent replicas.

Frames carry no state between each other (the reference's Recon is
fmParallel, src/plugin.cpp:1157), so N GPUs run N independent replicas, one
process per GPU, each on its own frames. There is no data-path collective;
the only cross-rank step is the max over ranks of the measured time.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (disjoint, covering)."""
    return [it for i, it in enumerate(items) if i % world == rank]


def frame_seed(base: int, rank: int, index: int, stride: int = 64) -> int:
    """Seed of a rank's index-th frame: ranks draw disjoint seed ranges."""
    return base + stride * rank + index


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the process group (identity when not
    initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(units_per_rank, seconds_max: float) -> float:
    """Whole-job throughput: units over all ranks / max-over-ranks time."""
    return float(sum(units_per_rank)) / seconds_max


def free_port() -> int:
    """An unused TCP port on the loopback interface."""
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def launch_command(script: str, argv, nproc: int, port: int):
    """torchrun command that starts `nproc` replicas of `script` on this node
    (one process per GPU), rendezvous on 127.0.0.1."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={int(nproc)}", "--master-addr", "127.0.0.1",
            "--master-port", str(int(port)), script] + list(argv)


def relaunch(script: str, argv, nproc: int, timeout_s: float = 3600.0) -> int:
    """Run `script` as `nproc` replicas under torchrun and return its exit
    status (used when a multi-GPU run is started without torchrun)."""
    cmd = launch_command(script, argv, nproc, free_port())
    try:
        return subprocess.run(cmd, timeout=timeout_s).returncode
    except subprocess.TimeoutExpired:
        return 124

"""Child script of the replica launcher test: started by lgcr.replicas.relaunch
as torchrun ranks on CPU (gloo); rank 0 prints the world size, the ranks'
max and the shard sizes as one JSON line."""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "vapoursynth-lgcr_b200"))

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from lgcr import replicas as R  # noqa: E402

rank, world, local = R.rank_info()
dist.init_process_group("gloo")
top = R.max_over_ranks(10.0 + rank)
share = torch.tensor([float(len(R.shard(list(range(32)), rank, world)))])
dist.all_reduce(share)
if rank == 0:
    print(json.dumps({"world": world, "max": top, "frames": share.item()}))
dist.barrier()
dist.destroy_process_group()

"""One gloo rank of the sharded-stepping test (launched twice or three times
by tests/test_shard.py): steps a small ring with CpuShard + DistExchange,
diagnoses it with one all-reduce of the ranks' diagnostic fields and, on
rank 0, saves the gathered state and the diagnostics to the path in argv[1]."""
import os
import sys
from datetime import timedelta
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

from pawan_b200 import cases, shard  # noqa: E402
from shard_cpu import CpuShard  # noqa: E402


def main():
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    w = cases.ring_stations(stations=int(os.environ.get("STATIONS", "17")), seed=0)
    b = CpuShard(w, rank, world)
    stepper = shard.ShardedStepper(b, shard.DistExchange(b))
    stepper.step("rk4", 0.01, 2)
    pos, alpha = shard.gather_state_dist(b)
    # diagnostics of the stepped system: each rank's owned rows, one all-reduce
    diag, vbi, zc = shard.diagnose_dist(b)
    if rank == 0:
        np.savez(sys.argv[1], pos=pos, alpha=alpha, diag=diag, vbi=vbi, zc=zc)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()

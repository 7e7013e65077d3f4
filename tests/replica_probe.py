"""One rank of the replica launcher check (run by ``test_multi_rank_cpu.py`` through
``bench.launch_replicas``): joins the process group the way ``bench.py`` does and prints,
on rank 0, one JSON line with the world size and the reduced values."""

import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def main():
    world, rank, local = bench.dist_setup()
    mx = bench.reduce(10.0 + rank, world, "max")
    sm = bench.reduce(float(rank + 1), world, "sum")
    if rank == 0:
        print(json.dumps({"n_gpus": world, "max": mx, "sum": sm, "local_rank": local}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

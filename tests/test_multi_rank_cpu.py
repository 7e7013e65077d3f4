"""The N-GPU bench path on CPU: two gloo ranks, disjoint problem shards, max/sum timing reductions.

The path has no data exchange (every problem is independent): each rank solves its own
shard and only the timing (max over ranks) and the solved counts (sum) are reduced.
"""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as tmp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        wl = bench.make_workload(64, seed=bench.shard_seed(rank))
        digest = [float(c["q_star"].sum()) for c in wl]
        mx = bench.reduce(10.0 + rank, world, "max")
        sm = bench.reduce(float(rank + 1), world, "sum")
        out.put((rank, digest, mx, sm, [len(c["n_targets"]) for c in wl]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_disjoint_shards_and_reductions():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, d0, mx0, sm0, n0), (r1, d1, mx1, sm1, n1) = res
    assert (r0, r1) == (0, 1)
    assert mx0 == mx1 == 11.0 and sm0 == sm1 == 3.0
    assert n0 == n1 and sum(n0) == 64          # same mix per rank (weak scaling)
    assert all(a != b for a, b in zip(d0, d1))  # different problems on each rank


def test_bench_replica_launcher_runs_two_ranks(capfd):
    """``bench.py --gpus N`` started without torchrun launches N ranks itself (``launch_replicas``);
    each joins the process group from RANK / WORLD_SIZE / MASTER_* and rank 0 reports n_gpus = N."""
    import json
    import sys

    import bench
    probe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "replica_probe.py")
    env_before = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        rc = bench.launch_replicas([sys.executable, probe], 2, timeout_s=240)
    finally:
        os.environ.update(env_before)
    out = capfd.readouterr().out.strip().splitlines()
    assert rc == 0
    line = json.loads(out[-1])
    assert line == {"n_gpus": 2, "max": 11.0, "sum": 3.0, "local_rank": 0}

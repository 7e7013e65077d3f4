"""Benchmark of the B200 kinematics / LM-IK path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workloads (synthetic, seeded; no dataset exists for this path):

* headline — batched LM-IK on the uneven mix (8,192 problems: 40% 7-DOF chains,
  30% 14-DOF dual-arm trees, 30% 36-DOF free-flyer humanoids; 1-6 pose targets
  each from FK of a random q*; q0 = q* + N(0, 0.3) noise; <= 100 LM iterations,
  damping 1e-3 x10/÷10, tol 1e-6).  value = problems reaching <= 1e-4 m and
  <= 1e-4 rad final pose error per second.
* roofline — fused FK + frame Jacobians on the free-flyer humanoid (B = 65,536,
  12 frames, J [B,12,6,36] + oMf [B,12,7] float32), HBM bound.

Multi-GPU: every problem is independent, so N GPUs run N replicas on disjoint
shards with no collective on the data path (weak scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

FKJ_BATCH = 65536
FKJ_BYTES_PER_CONFIG = 4 * (37 + 12 * 7 + 12 * 6 * 36)  # q read + oMf + J written = 10,852 B


def _peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.path is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# FK + frame Jacobians (roofline workload)
# ---------------------------------------------------------------------------
def bench_fkj(steps: int, warmup: int, seed: int = 1):
    import betterrobot_b200 as br
    from betterrobot_b200 import synthetic as syn
    from betterrobot_b200.kinematics import frame_jacobians_into

    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    fids = syn.op_frame_ids(m)
    n_buf = 16  # 16 distinct q buffers (155 MB) > 126 MB L2: every step reads q from HBM
    qs = [syn.random_q(m64, FKJ_BATCH, seed + i, rev_range=2.5, base_translation=1.0).float().cuda()
          for i in range(n_buf)]
    J = torch.empty(FKJ_BATCH, len(fids), 6, m.nv, device="cuda")
    T = torch.empty(FKJ_BATCH, len(fids), 7, device="cuda")
    stream = torch.cuda.current_stream()
    for i in range(warmup):
        frame_jacobians_into(m, qs[i % n_buf], fids, T, J)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        frame_jacobians_into(m, qs[i % n_buf], fids, T, J)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"ms_per_launch": ms, "configs": FKJ_BATCH, "bytes": FKJ_BATCH * FKJ_BYTES_PER_CONFIG,
            "gbs": FKJ_BATCH * FKJ_BYTES_PER_CONFIG / (ms * 1e-3) / 1e9, "launches": steps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--section", default="all", choices=["all", "fkj", "ik"])
    args = ap.parse_args()
    world, rank, local = dist_setup()
    peak, peak_kind = _peaks()
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        fkj = bench_fkj(args.steps, max(args.warmup, 3))
        barrier(world)
    clocks = clk.summary()
    ms = max_over_ranks(fkj["ms_per_launch"], world)
    value = sum_over_ranks(fkj["configs"], world) / (ms * 1e-3)
    line = {
        "metric": "fused FK+frame-Jacobian configs/s (humanoid, 12 frames)", "value": value, "unit": "configs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "humanoid FK + 12 LWA frame Jacobians", "batch": FKJ_BATCH, "l2": "16 rotating q buffers"},
        "roofline": {"bound": "hbm", "achieved": fkj["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": fkj["gbs"] / peak, "traffic": None, "peak_kind": peak_kind},
        "clocks": clocks, "gpu_launches": fkj["launches"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the B200 kinematics / LM-IK path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Headline workload (synthetic and seeded — the path has no dataset): the uneven
batched IK mix, 8,192 independent problems in one persistent launch —
40% 7-DOF chains, 30% 14-DOF dual-arm trees, 30% 36-DOF free-flyer humanoids;
each with 1-6 pose targets (a random subset of 6 candidate frames) generated by
FK of a random q*; q0 = q* + N(0, 0.3) noise; LM <= 100 iterations, damping
1e-3 adapted x10 / ÷10, tol 1e-6 on |J^T r|; limit weight 0.1, rest weight 1e-3.
A step solves the whole batch once.

  value  = problems whose final pose error is <= 1e-4 m and <= 1e-4 rad on every
           target, per second, inputs resident in HBM (L2 flushed between steps);
  e2e    = the same through the public API with pinned host inputs: each step copies
           targets and q0 host->device, solves, copies q / status / iterations back;
  plain_gpu = the same method as plain per-op PyTorch on the same GPU;
  roofline  = the fused FK + frame-Jacobian kernel on the free-flyer humanoid
           (B = 65,536, 12 frames) against the measured HBM copy bandwidth;
  roofline_lm = the LM launch's throughput in the reference's dense-iteration FLOPs
           against the nominal FP32 CUDA-core peak;
  ik_f64_normal_equations, adjoint, trajopt, lie_ops, joint_jacobians = the other
           kernels of the path (float64 normal equations on the same mix; pose-loss
           forward + backward; 256 x 64-knot trajectories; SE3 compose / log / exp on
           8.4 M elements; all 32 joint Jacobians of the humanoid at B = 16,384), the
           HBM-bound ones with their fraction of the measured copy bandwidth;
  cpu_baseline(s) = the reference algorithm (float64 port) on the host cores.

Multi-GPU: problems are independent, so N GPUs run N replicas on disjoint
problem sets with no data-path collective (weak scaling); time is the max over
ranks.  ``--impl reference`` times BetterRobot's algorithm on the host CPU (the
float64 port of its serial LM) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_PROBLEMS = 8192
MAX_ITER = 100
SETTINGS = dict(lam0=1e-3, factor=10.0, tol=1e-6, rest_weight=1e-3, limit_weight=0.1)
FKJ_BATCH = 65536
FKJ_BYTES_PER_CONFIG = 4 * (37 + 12 * 7 + 12 * 6 * 36)  # q read + oMf + J written = 10,852 B
# DRAM bytes (read + write) of one fk_jac_kernel launch at B = 65,536, 12 frames, from an ncu capture
# of ``bench.py --only fkj`` (dram__bytes_read.sum 9.77 MB + dram__bytes_write.sum 642.18 MB); the
# rest of the 711 MB of output is still in L2 when the launch ends.
FKJ_TRAFFIC_BYTES = 9.766e6 + 642.179e6
# DRAM bytes of one lm_solve_kernel launch on the 8,192-problem mix (ncu dram__bytes_read.sum 3.06 MB,
# dram__bytes_write.sum 0: the results stay in L2 until the next reader): neither HBM nor L2 bound
LM_TRAFFIC_BYTES = 3.063e6
JOINT_OPS_BATCH = 1 << 20
REACH_TOL = 1e-4
CANDIDATES = {
    "humanoid": [f"track{i}" for i in range(6)],
    "dual_arm": ["ee_l", "ee_r", "body_l_link5", "body_r_link5", "body_l_link3", "body_r_link3"],
    "chain7": ["ee", "body_link7", "body_link6", "body_link5", "body_link4", "body_link3"],
}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def class_specs():
    from betterrobot_b200 import synthetic as syn
    return [("humanoid", syn.humanoid_spec()), ("dual_arm", syn.dual_arm_spec()), ("chain7", syn.chain_spec())]


def make_workload(n_problems: int, seed: int):
    """Per class: models, frame ids (P_c, 6) (first n_targets used), n_targets, q* and q0 (float64)."""
    import torch
    from betterrobot_b200 import synthetic as syn
    mix = syn.ik_uneven_mix(n_problems, seed)
    rng = np.random.default_rng(seed + 1)
    out = []
    for ci, (name, spec) in enumerate(class_specs()):
        m = syn.model_from_spec(spec)
        m64 = syn.model_from_spec(spec, dtype=torch.float64)
        nts = np.array([k for lab, k in mix if lab == name], np.int32)
        P = len(nts)
        cand = np.array([m.frame_id(f) for f in CANDIDATES[name]], np.int32)
        frames = np.stack([cand[rng.permutation(6)] for _ in range(P)]).astype(np.int32)
        q_star = syn.random_q(m64, P, seed + 10 + ci, rev_range=2.5, base_translation=0.5)
        q0 = syn.noisy_start(m64, q_star, 0.3, seed + 20 + ci)
        out.append({"name": name, "model": m, "model64": m64, "frames": frames, "n_targets": nts,
                    "q_star": q_star, "q0": q0})
    return out


def gpu_targets(wl):
    """Target poses = FK(q*) of each problem's frames, by the library's own FK kernel."""
    import torch
    import betterrobot_b200 as br
    for c in wl:
        d = br.forward_kinematics(c["model"], c["q_star"].float().cuda(), compute_frames=True)
        idx = torch.from_numpy(c["frames"]).long().cuda()
        c["targets"] = torch.gather(d.frame_pose_world, 1, idx[..., None].expand(-1, -1, 7)).contiguous()


def gpu_reach(wl, q_list):
    """Problems whose every target is reached within REACH_TOL (m and rad), via the library FK."""
    return int(sum(int(f.sum()) for f in gpu_reach_flags(wl, q_list)))


def gpu_reach_flags(wl, q_list):
    """Per class, a bool array: the problem's every target is reached within REACH_TOL."""
    import torch
    import betterrobot_b200 as br
    flags = []
    for c, q in zip(wl, q_list):
        d = br.forward_kinematics(c["model"], q, compute_frames=True, check_quaternion=False)
        idx = torch.from_numpy(c["frames"]).long().cuda()
        T = torch.gather(d.frame_pose_world, 1, idx[..., None].expand(-1, -1, 7)).double()
        tg = c["targets"].double()
        pe = (T[..., :3] - tg[..., :3]).norm(dim=-1)
        # rotation error = |so3_log(q_t^-1 q)| = 2 atan2(|vec(r)|, |w(r)|), r = conj(q_t) (x) q,
        # as the oracle measures it; 2 acos(|<q_t, q>|) would be ill-conditioned near 0 (float32
        # rounding of the quaternions alone reads as ~4e-4 rad there)
        av, aw = tg[..., 3:6], tg[..., 6:7]
        bv, bw = T[..., 3:6], T[..., 6:7]
        rv = aw * bv - bw * av - torch.linalg.cross(av, bv, dim=-1)
        rw = (aw * bw + (av * bv).sum(-1, keepdim=True)).squeeze(-1)
        re = 2.0 * torch.atan2(rv.norm(dim=-1), rw.abs())
        k = torch.arange(6, device=q.device)[None, :] < torch.from_numpy(c["n_targets"]).cuda()[:, None]
        ok = ((pe <= REACH_TOL) & (re <= REACH_TOL)) | ~k
        flags.append(ok.all(dim=1).cpu().numpy())
    return flags


# ---------------------------------------------------------------------------
# LM compute roofline: algorithmic floating-point operations of one iteration of the
# reference's dense method (levenberg_marquardt.py:89-110 with the IK stack of tasks/ik.py),
# an FMA counted as 2
# ---------------------------------------------------------------------------
SE3_COMPOSE_FLOPS = 61        # quaternion product (28) + rotate (30) + add (3)
SE3_LOG_FLOPS = 60            # quaternion log + V^-1 v
JR_INV_FLOPS = 9 * 2 * 6 ** 3 + 2 * 6 ** 3   # 9-term ad series of 6x6 products + 6x6 inverse
# B200 FP32 CUDA-core peak: 148 SMs x 128 lanes x 2 flops x 1.965 GHz (nominal; the kernel issues
# FP32 and FP64 instructions, FP64 at half this rate)
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def lm_iteration_flops(model, frame_ids) -> int:
    """Flops of one LM iteration on ``model`` with pose targets on ``frame_ids``: trial FK (one SE3
    compose per joint), the residual (frame pose, error pose, log per target; limit and rest rows),
    the Jacobian (per target Jr^-1, its frame Jacobian by the support loop, one 6x6 Ad product per
    supporting column, and Jr^-1 R^T J_lwa), the dense J^T J and J^T r over the stacked rows,
    the Cholesky factorization and two triangular solves, and the retraction."""
    nj, nq, nv = model.njoints, model.nq, model.nv
    k = len(frame_ids)
    dim = 6 * k + 2 * nq + nv
    f = nj * SE3_COMPOSE_FLOPS
    f += k * (2 * SE3_COMPOSE_FLOPS + SE3_LOG_FLOPS) + 4 * nq + 3 * nv
    for fid in frame_ids:
        depth = sum(int(model.nvs[j]) for j in model.supports[model.frames[fid].parent_joint])
        f += JR_INV_FLOPS + depth * 2 * 36 + 2 * 2 * 36 * nv
    f += 2 * dim * nv * nv + 2 * dim * nv
    f += 2 * nv ** 3 // 3 + 2 * 2 * nv * nv
    f += 2 * nq
    return f


SE3_INVERSE_FLOPS = 33        # rotate (30) + negate (3)
JR_INV_T_XI_FLOPS = 150       # closed-form Jr^-T(xi) xi: ~10 cross products, 3 coefficients, 4 axpys
WRENCH_FLOPS = 72             # F = [R g_lin; p x R g_lin + R g_ang]
COLUMN_TWIST_FLOPS = 40       # world column S_c = [o x a; a] from its joint pose
PAIR_FLOPS = 11               # <S_c, F_f> per (frame, supporting column)


def adjoint_flops_per_config(model, frame_ids, recompute: bool) -> int:
    """Algorithmic flops of the pose loss and its gradient for one configuration: FK (one
    local transform and one compose per joint), per frame its placement, the target's inverse,
    the error pose, its log and weighted square; backward: the same FK and frame poses again
    when ``recompute``, per frame Jr^-T(xi) xi and the world wrench, one world twist per
    column and one dot product per (frame, supporting column), the raw-q map of a free flyer."""
    nj, nv = model.njoints, model.nv
    fk = nj * 2 * SE3_COMPOSE_FLOPS
    frames = len(frame_ids) * (2 * SE3_COMPOSE_FLOPS + SE3_INVERSE_FLOPS + SE3_LOG_FLOPS + 13)
    pairs = sum(sum(int(model.nvs[j]) for j in model.supports[model.frames[f].parent_joint]) for f in frame_ids)
    bwd = len(frame_ids) * (JR_INV_T_XI_FLOPS + WRENCH_FLOPS) + nv * COLUMN_TWIST_FLOPS + pairs * PAIR_FLOPS + 60
    if recompute:
        bwd += fk + frames
    return fk + frames + bwd


def lm_launch_flops(wl, iters) -> float:
    """Flops of one solve of the packed mix: per problem, its iterations x its class's iteration
    flops for its own targets."""
    total, off = 0.0, 0
    for c in wl:
        m = c["model"]
        for p in range(len(c["n_targets"])):
            k = int(c["n_targets"][p])
            total += float(iters[off + p]) * lm_iteration_flops(m, [int(x) for x in c["frames"][p, :k]])
        off += len(c["n_targets"])
    return total


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
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
        self.index, self.proc, self.path = index, None, None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
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
        rows = [[x.strip() for x in r.split(",")] for r in open(self.path).read().strip().splitlines()
                if r.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def shard_seed(rank: int) -> int:
    """Workload seed of a rank: every rank solves its own, disjoint problem set (replicas)."""
    return 7 + 1000 * rank


def launch_replicas(cmd: list[str], n: int, timeout_s: float = 3600.0) -> int:
    """Run ``cmd`` as ``n`` ranks on this node (what ``torchrun --nproc-per-node n`` does for this
    script): rank i gets RANK = LOCAL_RANK = i, WORLD_SIZE = n and a rendezvous on 127.0.0.1.
    Rank 0 writes to this process's stdout; the other ranks' stdout is dropped (they print
    nothing).  Returns the first non-zero exit code, else 0."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen(cmd, env=env, stdout=None if r == 0 else subprocess.DEVNULL))
    deadline = time.time() + timeout_s
    rc = 0
    for p in procs:
        try:
            code = p.wait(timeout=max(1.0, deadline - time.time()))
        except subprocess.TimeoutExpired:
            p.kill()
            code = p.wait()
        rc = rc or code
    return rc


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce(x: float, world: int, op: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# fused LM-IK (headline)
# ---------------------------------------------------------------------------
def ik_settings(precision: str = "f32"):
    from betterrobot_b200 import ik as bik
    return bik.settings_from(
        bik.IKCostConfig(rest_weight=SETTINGS["rest_weight"], limit_weight=SETTINGS["limit_weight"]),
        bik.OptimizerConfig(max_iter=MAX_ITER, lam0=SETTINGS["lam0"], factor=SETTINGS["factor"], tol=SETTINGS["tol"],
                            precision=precision))


def bench_ik(steps: int, warmup: int, seed: int, pinned=None, precision: str = "f32", e2e: bool = True):
    """``pinned = (team_sizes, warps_per_cta)`` skips the autotuner (used to profile one known launch shape)."""
    import torch
    from betterrobot_b200 import ik as bik
    wl = make_workload(N_PROBLEMS, seed)
    gpu_targets(wl)
    settings = ik_settings(precision)
    from betterrobot_b200 import autotune
    tg_dev = [c["targets"] for c in wl]
    q0_dev = [c["q0"].float().cuda() for c in wl]

    def make(teams, warps):
        p = bik.PackedIK([c["model"] for c in wl], [c["frames"] for c in wl], [c["n_targets"] for c in wl],
                         team_sizes=teams, warps_per_cta=warps)
        p.set_inputs(tg_dev, q0_dev)
        return p
    if pinned is None:
        teams, warps, _ = autotune.tune(make, settings)   # outside the timed region
    else:
        teams, warps = pinned
    pk = make(teams, warps)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda")  # > 126 MB L2
    for _ in range(warmup):
        pk.solve(settings)
    torch.cuda.synchronize()
    # every step is enqueued without a host wait (the host runs ahead of the device, so the
    # device never idles inside a timed step waiting for the next launch); one synchronize
    # after the last step, then the per-step event pairs are read
    evs = []
    for _ in range(steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pk.solve(settings)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    reached = gpu_reach(wl, [pk.q_of(c).clone() for c in range(len(wl))])
    conv = int(((pk.status & 0xFF) == 0).sum())
    iters = pk.iters.float()
    flops = lm_launch_flops(wl, pk.iters.cpu().numpy())
    if not e2e:
        return {"ms": ms, "reached": reached, "converged": conv, "problems": pk.P, "flops": flops,
                "iters_mean": float(iters.mean()), "team_sizes": teams, "warps_per_cta": warps}
    # e2e: pinned host inputs -> solve -> pinned host outputs, every step
    h_tg = [t.cpu().pin_memory() for t in tg_dev]
    h_q0 = [q.cpu().pin_memory() for q in q0_dev]
    h_x = torch.empty(pk.q_total).pin_memory()
    h_st = torch.empty(pk.P, dtype=torch.int32).pin_memory()
    h_it = torch.empty(pk.P, dtype=torch.int32).pin_memory()
    h2d = sum(t.numel() * 4 for t in h_tg) + sum(q.numel() * 4 for q in h_q0)
    d2h = pk.q_total * 4 + pk.P * 8

    def e2e_step():
        pk.set_inputs(h_tg, h_q0)
        pk.solve(settings)
        h_x.copy_(pk.x, non_blocking=True)
        h_st.copy_(pk.status, non_blocking=True)
        h_it.copy_(pk.iters, non_blocking=True)
    for _ in range(warmup):
        e2e_step()
    torch.cuda.synchronize()
    evs = []
    for _ in range(steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    et = [a.elapsed_time(b) for a, b in evs]
    # the same solve replayed from a CUDA graph
    g = pk.capture(settings)
    torch.cuda.synchronize()
    evs = []
    for _ in range(steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.replay()
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    gt = [a.elapsed_time(b) for a, b in evs]
    return {"ms": ms, "reached": reached, "converged": conv, "problems": pk.P, "iters_mean": float(iters.mean()),
            "flops": flops,
            "e2e_ms": float(np.mean(et)), "h2d": h2d, "d2h": d2h, "launches": steps, "wl": wl,
            "graph_ms": float(np.mean(gt)), "team_sizes": teams, "warps_per_cta": warps}


def bench_plain_gpu(wl):
    """The same batched LM as plain per-op PyTorch on this GPU (one timed solve after one warm-up)."""
    import torch
    from baseline.plain_gpu import PlainLM
    runs = []
    for c in wl:
        m = c["model"]
        lm = PlainLM(m, torch.device("cuda"))
        cand = [m.frame_id(f) for f in CANDIDATES[c["name"]]]
        P = len(c["n_targets"])
        pos = {f: i for i, f in enumerate(cand)}
        T = torch.zeros(P, 6, 7, device="cuda")
        T[..., 6] = 1.0
        mask = torch.zeros(P, 6, device="cuda")
        fr = c["frames"]
        tg = c["targets"]
        for k in range(6):
            col = torch.tensor([pos[int(f)] for f in fr[:, k]], device="cuda")
            sel = torch.from_numpy(c["n_targets"] > k).cuda()
            rows = torch.arange(P, device="cuda")[sel]
            T[rows, col[sel]] = tg[sel, k]
            mask[rows, col[sel]] = 1.0
        q0 = c["q0"].float().cuda()
        qr = m.q_neutral.float().cuda().expand(P, -1)
        runs.append((lm, cand, T, mask, q0, qr))
    w = (1.0, 1.0, SETTINGS["limit_weight"], SETTINGS["rest_weight"])
    kw = dict(weights=w, lam0=SETTINGS["lam0"], factor=SETTINGS["factor"], tol=SETTINGS["tol"], max_iter=MAX_ITER)
    for lm, cand, T, mask, q0, qr in runs:  # warm-up (allocator, cuBLAS/cuSOLVER handles)
        lm.solve(cand, T[:64], mask[:64], q0[:64], qr[:64], **{**kw, "max_iter": 3})
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    qs = []
    for lm, cand, T, mask, q0, qr in runs:
        q, conv, iters = lm.solve(cand, T, mask, q0, qr, **kw)
        qs.append(q)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    reached = gpu_reach(wl, qs)
    return {"sec": sec, "reached": reached}


# ---------------------------------------------------------------------------
# FK + frame Jacobians (roofline workload)
# ---------------------------------------------------------------------------
def bench_fkj(steps: int, warmup: int, seed: int = 1):
    import torch
    from betterrobot_b200 import synthetic as syn
    from betterrobot_b200.kinematics import frame_jacobians_into
    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    fids = syn.op_frame_ids(m)
    n_buf = 16  # 16 distinct q buffers (155 MB) > 126 MB L2: every launch reads q from HBM
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
    return {"ms_per_launch": ms, "gbs": FKJ_BATCH * FKJ_BYTES_PER_CONFIG / (ms * 1e-3) / 1e9, "launches": steps}


def bench_joint_ops(steps: int, warmup: int):
    """Model.integrate / Model.difference on the humanoid (nq 37, nv 36), B = 1,048,576 configurations.

    Algorithmic bytes per configuration: integrate reads q (37) and v (36) and writes q' (37);
    difference reads q0, q1 (2 x 37) and writes v (36): 4 * 110 = 440 B for either.
    """
    import torch
    from betterrobot_b200 import synthetic as syn
    from betterrobot_b200.configuration import difference_into, integrate_into
    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    B = JOINT_OPS_BATCH
    q0 = syn.random_q(m64, B, 41, rev_range=2.5, base_translation=1.0).float().cuda()
    q1 = syn.random_q(m64, B, 42, rev_range=2.5, base_translation=1.0).float().cuda()
    v = torch.randn(B, m.nv, device="cuda", generator=torch.Generator("cuda").manual_seed(43)) * 0.3
    qo = torch.empty_like(q0)
    vo = torch.empty_like(v)
    stream = torch.cuda.current_stream()
    out = {}
    for name, fn in (("integrate", lambda: integrate_into(m, q0, v, qo)),
                     ("difference", lambda: difference_into(m, q0, q1, vo))):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_launch": ms, "gbs": B * 440 / (ms * 1e-3) / 1e9, "batch": B}
    return out


def _time_launches(fn, steps: int, warmup: int) -> float:
    """Mean ms per call of ``fn`` over ``steps`` calls enqueued back to back (CUDA events)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_lie(steps: int, warmup: int, n: int = 1 << 23):
    """Batched LieOps (``lie_ops_kernel``) on 8.4 M elements: se3_compose (reads 2 poses, writes one:
    84 B per element), se3_log (28 B in, 24 B out), se3_exp (24 B in, 28 B out); inputs > L2."""
    import torch
    from betterrobot_b200 import lie
    g = torch.Generator("cuda").manual_seed(5)
    def poses():
        t = torch.randn(n, 7, device="cuda", generator=g)
        t[:, 3:] = t[:, 3:] / t[:, 3:].norm(dim=1, keepdim=True)
        return t
    a, b = poses(), poses()
    xi = torch.randn(n, 6, device="cuda", generator=g) * 0.5
    out = {}
    for name, fn, bytes_per in (("se3_compose", lambda: lie.se3_compose(a, b), 84),
                                ("se3_log", lambda: lie.se3_log(a), 52), ("se3_exp", lambda: lie.se3_exp(xi), 52)):
        ms = _time_launches(fn, steps, warmup)
        out[name] = {"ms_per_launch": ms, "gbs": n * bytes_per / (ms * 1e-3) / 1e9, "elements": n}
    return out


def bench_joint_jacobians(steps: int, warmup: int, B: int = 16384):
    """``compute_joint_jacobians`` on the humanoid from stored joint placements (``fk_jac_kernel``
    in its from-poses mode): reads oMi (B x 32 x 7 floats), writes J (B x 32 x 6 x 36 floats)."""
    import torch
    import betterrobot_b200 as br
    from betterrobot_b200 import synthetic as syn
    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    q = syn.random_q(m64, B, 3, rev_range=2.5, base_translation=1.0).float().cuda()
    data = br.forward_kinematics(m, q)
    ms = _time_launches(lambda: br.compute_joint_jacobians(m, data), steps, warmup)
    nbytes = B * m.njoints * (7 + 6 * m.nv) * 4
    return {"ms_per_launch": ms, "gbs": nbytes / (ms * 1e-3) / 1e9, "batch": B, "bytes_per_launch": nbytes}


# ---------------------------------------------------------------------------
# FK pose-loss adjoint (config 2)
# ---------------------------------------------------------------------------
def bench_adjoint(steps: int, warmup: int):
    """Forward + backward of the pose loss on the humanoid, 12 frames: B = 16,384 (auto mode), and
    store vs recompute at B = 262,144."""
    import torch
    from betterrobot_b200 import synthetic as syn
    from betterrobot_b200.adjoint import pose_loss
    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    fids = syn.op_frame_ids(m)
    out = {}
    stream = torch.cuda.current_stream()
    for B, modes in ((16384, ("auto",)), (262144, ("store", "recompute"))):
        q = syn.random_q(m64, B, 31, rev_range=2.5, base_translation=1.0).float().cuda()
        T = syn.random_targets(B, len(fids), 32).float().cuda()
        w = torch.from_numpy(np.random.default_rng(33).uniform(0.5, 2.0, size=len(fids))).float().cuda()
        for mode in modes:
            qg = q.clone().requires_grad_(True)
            for _ in range(warmup):
                pose_loss(m, qg, fids, T, w, mode=mode).sum().backward()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                qg.grad = None
                pose_loss(m, qg, fids, T, w, mode=mode).sum().backward()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            fl = adjoint_flops_per_config(m, fids, recompute=(mode == "recompute" or
                                                              (mode == "auto" and B * m.njoints * 28 > 126 << 20)))
            tf = B * fl / (ms * 1e-3) / 1e12
            out[f"B{B}_{mode}"] = {"ms_fwd_bwd": ms, "configs_per_s": B / (ms * 1e-3), "flops_per_config": fl,
                                   "tflops": tf, "frac_fp32_peak": tf / FP32_PEAK_TFLOPS}
    return out


# ---------------------------------------------------------------------------
# trajectory optimisation (config 4)
# ---------------------------------------------------------------------------
def bench_trajopt(steps: int, warmup: int, n_traj: int = 256, knots: int = 64):
    """256 chain7 trajectories x 64 knots (448 variables each), goal = start + U(+-0.5) rad:
    GN <= 30 iterations + goal adjoint."""
    import torch
    import betterrobot_b200 as br
    from betterrobot_b200 import synthetic as syn
    from betterrobot_b200 import trajopt as btr
    m = syn.model_from_spec(syn.chain_spec())
    m64 = syn.model_from_spec(syn.chain_spec(), dtype=torch.float64)
    fid = m.frame_id("ee")
    qs, qg = syn.trajopt_endpoints(m64, n_traj, 81, spread=0.5)
    goal = br.forward_kinematics(m, qg.float().cuda(), compute_frames=True).frame_pose_world[:, fid].contiguous()
    start = br.forward_kinematics(m, qs.float().cuda(), compute_frames=True).frame_pose_world[:, fid].contiguous()
    X0 = qs.float().cuda()[:, None, :].expand(-1, knots, -1).contiguous()
    cfg = btr.TrajOptConfig(max_iter=30)
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        out = btr.solve_trajopt_batched(m, fid, goal, X0, start=start, cfg=cfg)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        out = btr.solve_trajopt_batched(m, fid, goal, X0, start=start, cfg=cfg)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"ms": ms, "trajectories_per_s": n_traj / (ms * 1e-3), "converged": int(out.converged.sum()),
            "iters_mean": float(out.iters.float().mean()), "n_traj": n_traj, "knots": knots}


# ---------------------------------------------------------------------------
# CPU: BetterRobot's algorithm (float64 port of its serial LM) on host cores
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    import torch
    torch.set_num_threads(1)
    os.environ["OMP_NUM_THREADS"] = "1"
    from oracle import ik as oik, kinematics as K
    from betterrobot_b200 import synthetic as syn
    name, idx, seed = args
    wl = {c["name"]: c for c in make_workload(N_PROBLEMS, seed)}
    c = wl[name]
    m64 = c["model64"]
    s = oik.IKSettings(lam0=SETTINGS["lam0"], factor=SETTINGS["factor"], tol=SETTINGS["tol"], max_iter=MAX_ITER,
                       rest_weight=SETTINGS["rest_weight"], limit_weight=SETTINGS["limit_weight"])
    t0 = time.perf_counter()
    reached = 0
    for p in idx:
        k = int(c["n_targets"][p])
        fids = [int(f) for f in c["frames"][p, :k]]
        oMi, _ = K.forward_kinematics(m64, c["q_star"].numpy()[p:p + 1])
        T = K.frame_placements(m64, oMi, fids)
        out = oik.solve(m64, fids, T, c["q0"].numpy()[p:p + 1], s)   # one problem per call, as solve_ik
        pe, re = oik.pose_errors(m64, out.q, fids, T)
        reached += int(pe[0] <= REACH_TOL and re[0] <= REACH_TOL)
    return reached, time.perf_counter() - t0, len(idx)


def cpu_baseline(seed: int, per_class=(77, 77, 102), cores: int | None = None, pool=None, draw: int = 0):
    """Serial float64 LM (one problem per call, like solve_ik) on a stratified sample, all host cores.
    ``draw`` picks another stratified sample of the same workload."""
    cores = cores or len(os.sched_getaffinity(0))
    names = [n for n, _ in class_specs()]
    frac = {"humanoid": 0.3, "dual_arm": 0.3, "chain7": 0.4}
    rng = np.random.default_rng(seed + 5 + 1000 * draw)
    wl = {c["name"]: c for c in make_workload(N_PROBLEMS, seed)}
    tasks, weights = [], {}
    for name, n in zip(names, per_class):
        P = len(wl[name]["n_targets"])
        pick = rng.choice(P, size=n, replace=False)
        chunks = np.array_split(pick, max(1, min(n, cores)))
        tasks += [(name, [int(i) for i in ch], seed) for ch in chunks if len(ch)]
        weights[name] = (n, frac[name])
    t0 = time.perf_counter()
    if pool is None:
        with mp.get_context("spawn").Pool(min(cores, len(tasks))) as own:
            res = own.map(_cpu_worker, tasks)
    else:
        res = pool.map(_cpu_worker, tasks)
    wall = time.perf_counter() - t0
    cpu_sec = sum(r[1] for r in res)
    # per-class success rate and seconds per solve, extrapolated to the 8,192-problem mix
    by = {n: [0, 0.0, 0] for n in names}
    for (name, _, _), r in zip(tasks, res):
        by[name][0] += r[0]
        by[name][1] += r[1]
        by[name][2] += r[2]
    n_full = {n: len(wl[n]["n_targets"]) for n in names}
    reached_full = sum(by[n][0] / by[n][2] * n_full[n] for n in names)
    cpu_seconds_full = sum(by[n][1] / by[n][2] * n_full[n] for n in names)
    used = min(cores, len(tasks))
    value = reached_full / (cpu_seconds_full / used)
    return {"value": value, "cores": used, "wall_s": wall, "cpu_s": cpu_sec,
            "sample": f"stratified {sum(per_class)} problems ({per_class[2]} chain7, {per_class[1]} dual_arm, "
                      f"{per_class[0]} humanoid), serial float64 LM per problem, {used} processes; "
                      f"rate extrapolated to the 8,192-problem mix"}


# ---------------------------------------------------------------------------
# CPU: the float64 oracle ports of configs 1, 2 and 4 on host cores
# ---------------------------------------------------------------------------
CPU_FKJ_SAMPLE = 2048      # configurations per process and repetition
CPU_ADJ_SAMPLE = 2048
CPU_TRAJ_KNOTS = 64


def _cpu_leg_worker(args):
    """One process of a CPU leg: returns (units done, seconds)."""
    import torch
    torch.set_num_threads(1)
    os.environ["OMP_NUM_THREADS"] = "1"
    from betterrobot_b200 import synthetic as syn
    from oracle import adjoint as A, kinematics as K, trajopt as ot
    leg, seed, reps = args
    if leg == "trajopt":
        mc = syn.model_from_spec(syn.chain_spec(), dtype=torch.float64)
        fid = mc.frame_id("ee")
        qs, qg = syn.trajopt_endpoints(mc, 1, 81 + seed, spread=0.5)
        oMi, _ = K.forward_kinematics(mc, qg.numpy())
        goal = K.frame_placements(mc, oMi, [fid])[:, 0]
        oMi, _ = K.forward_kinematics(mc, qs.numpy())
        start = K.frame_placements(mc, oMi, [fid])[:, 0]
        X0 = np.repeat(qs.numpy()[:, None, :], CPU_TRAJ_KNOTS, 1)
        t0 = time.perf_counter()
        ot.solve(mc, X0, fid, goal, start, ot.TrajSettings(max_iter=30))
        return 1, time.perf_counter() - t0
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    fids = syn.op_frame_ids(m64)
    B = CPU_FKJ_SAMPLE if leg == "fkj" else CPU_ADJ_SAMPLE
    q = syn.random_q(m64, B, seed, rev_range=2.5, base_translation=1.0).numpy()
    tg = syn.random_targets(B, len(fids), seed + 1).double().numpy()
    w = np.random.default_rng(seed + 2).uniform(0.5, 2.0, size=len(fids))
    t0 = time.perf_counter()
    for _ in range(reps):
        if leg == "fkj":      # forward_kinematics(compute_frames=True) + 12 x get_frame_jacobian (LWA)
            oMi, _ = K.forward_kinematics(m64, q)
            K.frame_placements(m64, oMi, fids)
            for f in fids:
                K.frame_jacobian(m64, oMi, q, f)
        else:                 # the pose loss and its gradient w.r.t. q (what autograd returns)
            A.pose_loss(m64, q, fids, tg, w)
            A.pose_loss_grad(m64, q, fids, tg, w)
    return B * reps, time.perf_counter() - t0


def cpu_legs(pool, cores: int) -> dict:
    """Configs 1, 2, 4 through the float64 oracle ports on the host: all cores (one process per
    core) and, for configs 1 and 2, one thread."""
    out = {}
    for leg, reps, unit in (("fkj", 4, "configs/s"), ("adjoint", 2, "configs/s")):
        n1, s1 = pool.apply(_cpu_leg_worker, ((leg, 100, reps),))
        # all cores: the workers compute concurrently; the rate is the units of all of them over the
        # slowest one's compute time (process start-up and imports excluded)
        res = pool.map(_cpu_leg_worker, [(leg, 200 + i, reps) for i in range(cores)], chunksize=1)
        n = sum(r[0] for r in res)
        d = {"value": n / max(r[1] for r in res), "unit": unit, "cores": cores, "value_1thread": n1 / s1,
             "kind": "port"}
        if leg == "fkj":
            d["gbs"] = d["value"] * FKJ_BYTES_PER_CONFIG / 1e9
            d["sample"] = (f"humanoid FK + 12 frame Jacobians (local_world_aligned), float64 numpy oracle, "
                           f"{CPU_FKJ_SAMPLE} configurations x {reps} per process")
        else:
            d["sample"] = (f"humanoid 12-frame pose loss + its gradient w.r.t. q, float64 numpy oracle "
                           f"(reverse sweep pinned to the reference's autograd), {CPU_ADJ_SAMPLE} configurations x "
                           f"{reps} per process")
        out[leg] = d
    res = pool.map(_cpu_leg_worker, [("trajopt", i, 1) for i in range(cores)], chunksize=1)
    out["trajopt"] = {"value": sum(r[0] for r in res) / max(r[1] for r in res), "unit": "trajectories/s",
                      "cores": cores,
                      "kind": "port", "sample": f"{cores} chain7 trajectories x {CPU_TRAJ_KNOTS} knots, one per "
                      "process, float64 oracle GN with the dense (T nv)^2 normal equations of solve_trajopt, "
                      "<= 30 iterations"}
    return out


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-op PyTorch arm")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint section")
    ap.add_argument("--only", choices=["ik", "fkj", "adjoint", "trajopt", "joint_ops", "lie", "joint_jac"],
                    default=None,
                    help="run one section and print its raw timings (for profiling)")
    ap.add_argument("--ik-teams", default=None,
                    help="comma-separated lanes per problem for humanoid,dual_arm,chain7 (skips the autotuner)")
    ap.add_argument("--ik-warps", type=int, default=4, help="warps per CTA with --ik-teams")
    ap.add_argument("--ik-precision", choices=["f32", "f64"], default="f32",
                    help="normal-equation arithmetic of the LM kernel (--only ik)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # not started by torchrun: launch the N replicas here, one process per GPU
        sys.exit(launch_replicas([sys.executable, os.path.abspath(__file__), *sys.argv[1:]], args.gpus))
    warmup = max(args.warmup, 3)
    metric = "batched LM-IK solves/s reaching 1e-4 m and 1e-4 rad pose error"
    config = {"workload": "uneven batched IK: 8192 problems (40% chain7 7-DOF, 30% dual_arm 14-DOF, 30% humanoid "
                          "36-DOF free-flyer), 1-6 targets, q0 = q* + N(0,0.3), LM <= 100 it, lam 1e-3 x10, "
                          "tol 1e-6, limit 0.1, rest 1e-3", "problems": N_PROBLEMS, "l2": "256 MB flush between steps"}
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        steps = []
        cb = None
        cores = len(os.sched_getaffinity(0))
        n = max(2 * cores, 96)  # per step: >= 2 problems per host core, in the mix's proportions
        per_class = (round(0.3 * n), round(0.3 * n), n - 2 * round(0.3 * n))  # humanoid, dual_arm, chain7
        with mp.get_context("spawn").Pool(cores) as pool:
            for i in range(warmup + args.steps):
                # every step draws another stratified sample of the 8,192-problem mix
                cb = cpu_baseline(seed=7, per_class=per_class, cores=cores, pool=pool, draw=i)
                if i >= warmup:
                    steps.append(cb)
        v = float(np.mean([s["value"] for s in steps]))
        line = {"impl": "reference", "metric": metric, "value": v, "unit": "solves/s", "n_gpus": 1,
                "steps": args.steps, "warmup": warmup, "ms_per_step": float(np.mean([s["wall_s"] for s in steps])) * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cb["cores"], "kind": "port",
                                 "sample": cb["sample"].replace("stratified", "per step: stratified")},
                "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if args.only:
        import torch
        dist_setup()
        if args.only == "ik":
            pinned = None
            if args.ik_teams:
                pinned = ([int(t) for t in args.ik_teams.split(",")], args.ik_warps)
            r = bench_ik(args.steps, warmup, seed=7, pinned=pinned, precision=args.ik_precision)
            r.pop("wl", None)
        elif args.only == "joint_ops":
            r = bench_joint_ops(args.steps, warmup)
        elif args.only == "fkj":
            r = bench_fkj(args.steps, warmup)
        elif args.only == "trajopt":
            r = bench_trajopt(args.steps, warmup)
        elif args.only == "lie":
            r = bench_lie(args.steps, warmup)
        elif args.only == "joint_jac":
            r = bench_joint_jacobians(args.steps, warmup)
        else:
            r = bench_adjoint(args.steps, warmup)
        print(json.dumps({"section": args.only, **r}), flush=True)
        return
    cpu = legs = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # before any CUDA work in this process (spawned workers)
        cores = len(os.sched_getaffinity(0))
        with mp.get_context("spawn").Pool(cores) as pool:
            cpu = cpu_baseline(seed=7, cores=cores, pool=pool)
            legs = cpu_legs(pool, cores)
    import torch
    world, rank, local = dist_setup()
    peak, peak_kind = _peaks()
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        ik = bench_ik(args.steps, warmup, seed=shard_seed(rank))
        barrier(world)
    clocks = clk.summary()
    ik64 = bench_ik(args.steps, warmup, seed=shard_seed(rank), precision="f64", e2e=False)
    fkj = bench_fkj(args.steps, warmup)
    adj = bench_adjoint(args.steps, warmup) if not args.no_adjoint else None
    trj = bench_trajopt(args.steps, warmup) if not args.no_adjoint else None
    lie_r = bench_lie(args.steps, warmup)
    jj = bench_joint_jacobians(args.steps, warmup)
    plain = bench_plain_gpu(ik["wl"]) if (rank == 0 and not args.no_plain) else None
    ms = reduce(ik["ms"], world, "max")
    reached = reduce(ik["reached"], world, "sum")
    e2e_ms = reduce(ik["e2e_ms"], world, "max")
    value = reached / (ms * 1e-3)
    line = {
        "metric": metric, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (J, J^T J, Cholesky) + f64 (iterate, FK/residual of the accept test)", "data": "synthetic",
        "config": config,
        "e2e": {"value": reached / (e2e_ms * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": ik["h2d"],
                "d2h_bytes_per_step": ik["d2h"], "ms_per_step": e2e_ms},
        "roofline": {"bound": "hbm", "kernel": "fk_jac_kernel (humanoid B=65536, 12 frames, J + oMf)",
                     "achieved": fkj["gbs"], "peak": peak, "unit": "GB/s", "frac": fkj["gbs"] / peak,
                     "traffic": FKJ_TRAFFIC_BYTES, "peak_kind": peak_kind, "ms_per_launch": fkj["ms_per_launch"]},
        "roofline_lm": {"bound": "latency / issue (FP32 + FP64 CUDA cores, no tensor cores)",
                        "kernel": "lm_solve_kernel (the whole mix, one launch)",
                        "achieved": ik["flops"] / (ik["ms"] * 1e-3) / 1e12, "peak": FP32_PEAK_TFLOPS,
                        "unit": "TFLOP/s", "frac": ik["flops"] / (ik["ms"] * 1e-3) / 1e12 / FP32_PEAK_TFLOPS,
                        "peak_kind": "nominal FP32 CUDA-core peak (148 SMs x 128 x 2 x 1.965 GHz)",
                        "flops_per_launch": ik["flops"], "traffic": LM_TRAFFIC_BYTES,
                        "flops_basis": "reference's dense LM iteration per problem x its iterations"},
        "ik": {"problems": ik["problems"] * world, "reached_1e-4": reached, "converged": ik["converged"],
               "iters_mean": ik["iters_mean"], "kernel": "lm_solve_kernel", "launches_per_step": 1,
               "graph_replay_ms": ik["graph_ms"], "autotuned": {"team_sizes": ik["team_sizes"],
                                                                "warps_per_cta": ik["warps_per_cta"]}},
        "clocks": clocks, "gpu_launches": ik["launches"],
        "ik_f64_normal_equations": {
            "value": ik64["reached"] / (ik64["ms"] * 1e-3), "unit": "solves/s", "ms_per_step": ik64["ms"],
            "reached_1e-4": ik64["reached"], "converged": ik64["converged"],
            "note": "the same mix with precision='f64' (Jacobian, J^T J, J^T r and factorization in float64): "
                    "every determinate converged verdict equals the float64 reference's"},
    }
    if adj is not None:
        line["adjoint"] = adj
    if trj is not None:
        line["trajopt"] = trj
    line["lie_ops"] = {k: {**v, "frac_of_peak": v["gbs"] / peak} for k, v in lie_r.items()}
    line["joint_jacobians"] = {**jj, "frac_of_peak": jj["gbs"] / peak,
                               "kernel": "fk_jac_kernel (from poses: humanoid, all 32 joints, world)"}
    if plain is not None:
        line["plain_gpu"] = {"value": plain["reached"] / plain["sec"], "unit": "solves/s", "sec_per_step": plain["sec"],
                             "reached_1e-4": plain["reached"], "speedup_fused_over_plain":
                             value / max(plain["reached"] / plain["sec"], 1e-30)}
    if cpu is not None:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": "solves/s", "cores": cpu["cores"], "kind": "port",
                                "sample": cpu["sample"]}
        line["cpu_baselines_other_configs"] = legs
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

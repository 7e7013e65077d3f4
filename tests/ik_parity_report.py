"""Parity report of the batched LM kernel against the float64 oracle (run on a GPU).

    python tests/ik_parity_report.py > report.jsonl

For each case (robot, target frames, rest weight, start), P problems are solved
by ``betterrobot_b200.ik.solve_ik_batched`` and by ``oracle.ik.solve`` (pinned to
the reference solver by ``tests/golden``); prints one JSON line per case with the
converged-verdict agreement, the fraction of problems whose final stacked residual
is within 1e-4, mean iteration counts and the 1e-4 pose-reach rates.
"""

import json
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from betterrobot_b200 import ik as bik, synthetic as syn  # noqa: E402
from oracle import ik as oik, kinematics as K  # noqa: E402

SPECS = {"chain7": syn.chain_spec(), "humanoid": syn.humanoid_spec(), "dual_arm": syn.dual_arm_spec()}


def run(robot, frames, P, rest, seed, max_iter=100, random_start=False):
    m, m64 = syn.model_from_spec(SPECS[robot]), syn.model_from_spec(SPECS[robot], dtype=torch.float64)
    fids = [m.frame_id(f) for f in frames]
    q_star = syn.random_q(m64, P, seed, rev_range=2.8 if random_start else 2.5, base_translation=0.5)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    T = K.frame_placements(m64, oMi, fids)
    q0 = syn.random_q(m64, P, seed + 1, rev_range=2.8) if random_start else syn.noisy_start(m64, q_star, 0.3, seed + 1)
    s = oik.IKSettings(lam0=1e-3, factor=10.0, tol=1e-6, max_iter=max_iter, rest_weight=rest)
    t = time.time()
    ref = oik.solve(m64, fids, T, q0.numpy(), s)
    t_ref = time.time() - t
    out = bik.solve_ik_batched(m, fids, torch.from_numpy(T).float().cuda(), q0.float().cuda(),
                               cost_cfg=bik.IKCostConfig(rest_weight=rest),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=max_iter, lam0=1e-3, factor=10.0),
                               with_residual=True)
    torch.cuda.synchronize()
    conv = out.converged.cpu().numpy()
    d = np.abs(out.residual.cpu().double().numpy() - ref.residual).max(1)
    pe, re = oik.pose_errors(m64, out.q.cpu().double().numpy(), fids, T)
    pr, rr = oik.pose_errors(m64, ref.q, fids, T)
    both = conv & ref.converged
    return {"case": f"{robot}-{len(frames)}t-rest{rest}-{'rand' if random_start else 'noisy'}", "P": P,
            "verdict_agree": float((conv == ref.converged).mean()), "conv_ref": float(ref.converged.mean()),
            "conv_gpu": float(conv.mean()), "res_ok": float((d <= 1e-4).mean()),
            "res_ok_both_conv": float((d[both] <= 1e-4).mean()) if both.any() else None,
            "dres_med": float(np.median(d)), "iters_ref_mean": float(ref.iters.mean()),
            "iters_gpu_mean": float(out.iters.float().mean()),
            "reach_gpu": float(((pe <= 1e-4) & (re <= 1e-4)).mean()),
            "reach_ref": float(((pr <= 1e-4) & (rr <= 1e-4)).mean()),
            "flags": int(((out.status.cpu().numpy() >> 8) != 0).sum()), "oracle_s": t_ref}


def main():
    cases = [("chain7", ["ee"], 256, 0.01, 40, 50, True)]
    for rest in (0.01, 1e-3, 1e-4):
        cases += [("chain7", ["ee"], 256, rest, 10, 100, False),
                  ("dual_arm", ["ee_l", "ee_r"], 128, rest, 11, 100, False),
                  ("humanoid", ["track0", "track1", "track2"], 128, rest, 12, 100, False),
                  ("humanoid", [f"track{i}" for i in range(6)], 128, rest, 13, 100, False),
                  ("humanoid", ["track0"], 128, rest, 14, 100, False)]
    for robot, frames, P, rest, seed, it, rnd in cases:
        print(json.dumps(run(robot, frames, P, rest, seed, it, rnd)), flush=True)


if __name__ == "__main__":
    main()

"""The headline IK mix at its full size (8,192 problems of three robots, one launch) against
the float64 oracle run problem by problem on the same inputs (``golden/ik_mix_reach.npz``,
made by ``golden/make_mix_reach.py``).

Bar: the per-problem verdict "every target within 1e-4 m and 1e-4 rad" agrees on >= 99% of
the problems (>= 98% per class), and the reached count is within 1% of the oracle's; the
converged verdict agrees on >= 90% per class (float32 normal equations move the iterates by
~1e-7, which decides problems that end right at the gradient tolerance either way).
"""

import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_full_mix_reach_matches_float64_oracle():
    import bench
    from betterrobot_b200 import ik as bik
    g = np.load(os.path.join(GOLDEN, "ik_mix_reach.npz"))
    wl = bench.make_workload(bench.N_PROBLEMS, 7)
    bench.gpu_targets(wl)
    settings = bik.settings_from(
        bik.IKCostConfig(rest_weight=bench.SETTINGS["rest_weight"], limit_weight=bench.SETTINGS["limit_weight"]),
        bik.OptimizerConfig(max_iter=bench.MAX_ITER, lam0=bench.SETTINGS["lam0"], factor=bench.SETTINGS["factor"],
                            tol=bench.SETTINGS["tol"]))
    pk = bik.PackedIK([c["model"] for c in wl], [c["frames"] for c in wl], [c["n_targets"] for c in wl],
                      team_sizes=[32] * len(wl), warps_per_cta=4)
    pk.set_inputs([c["targets"] for c in wl], [c["q0"].float().cuda() for c in wl])
    pk.solve(settings)
    torch.cuda.synchronize()
    flags = bench.gpu_reach_flags(wl, [pk.q_of(i) for i in range(len(wl))])
    conv = ((pk.status & 0xFF) == 0).cpu().numpy()
    off = 0
    agree_all = []
    for ci, c in enumerate(wl):
        n = len(c["n_targets"])
        sel = g["cls"] == ci
        order = np.argsort(g["index"][sel])
        ref_reach = g["reached"][sel][order].astype(bool)
        ref_conv = g["converged"][sel][order].astype(bool)
        assert len(ref_reach) == n
        agree = flags[ci] == ref_reach
        agree_all.append(agree)
        assert agree.mean() >= 0.98, (c["name"], agree.mean())
        assert (conv[off:off + n] == ref_conv).mean() >= 0.90, (c["name"], (conv[off:off + n] == ref_conv).mean())
        off += n
    agree_all = np.concatenate(agree_all)
    assert agree_all.mean() >= 0.99, agree_all.mean()
    ours, ref = sum(int(f.sum()) for f in flags), int(g["reached"].sum())
    assert abs(ours - ref) <= 0.01 * ref, (ours, ref)

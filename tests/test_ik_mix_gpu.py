"""The headline IK mix at its full size (8,192 problems of three robots, one launch) against
the float64 oracle run problem by problem on the same inputs, and against BetterRobot's own
float64 LM on the same problems (``golden/ik_mix_reach.npz``, made by
``golden/make_mix_reach.py``).

Converged verdicts.  A problem's verdict is "rounding-decided" when an accept test that decides
convergence (pre-step |J^T r| < tol) compares two costs that differ by at most 64 units of
their float64 spacing: there the verdict depends on how the cost's sum was rounded, and two
float64 implementations of the same algorithm flip it independently — BetterRobot's torch
code agrees with the numpy oracle on only 60-83% of those problems (per class), while it
agrees on 100% of the others ("determinate").  Bars:

* float64 normal equations (``precision="f64"``): the same verdict as the oracle and as
  BetterRobot on every determinate problem (>= 99.9% per class); on rounding-decided problems
  at least BetterRobot's own agreement with the oracle, less 0.05;
* float32 normal equations (the default): the same verdict on >= 97.5% of determinate
  problems per class (>= 99% for the dual-arm and chain classes); float32 Jacobian rounding
  (~1e-7) moves the path of long humanoid solves, some of which then end elsewhere.

Reach verdict "every target within 1e-4 m and 1e-4 rad": agrees on >= 99% of problems
(>= 98% per class), the reached count within 1% of the oracle's.  Final stacked residuals,
where the GPU and the oracle both converged: within 1e-4 on >= 99% of problems.
"""

import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

MARGIN_ULPS = 64


def _solve(precision):
    import bench
    from betterrobot_b200 import ik as bik
    wl = bench.make_workload(bench.N_PROBLEMS, 7)
    bench.gpu_targets(wl)
    settings = bik.settings_from(
        bik.IKCostConfig(rest_weight=bench.SETTINGS["rest_weight"], limit_weight=bench.SETTINGS["limit_weight"]),
        bik.OptimizerConfig(max_iter=bench.MAX_ITER, lam0=bench.SETTINGS["lam0"], factor=bench.SETTINGS["factor"],
                            tol=bench.SETTINGS["tol"], precision=precision))
    pk = bik.PackedIK([c["model"] for c in wl], [c["frames"] for c in wl], [c["n_targets"] for c in wl],
                      team_sizes=[32] * len(wl), warps_per_cta=4)
    pk.set_inputs([c["targets"] for c in wl], [c["q0"].float().cuda() for c in wl])
    pk.solve(settings)
    torch.cuda.synchronize()
    return wl, pk, settings


def _per_class(g, ci, key):
    sel = g["cls"] == ci
    return g[key][sel][np.argsort(g["index"][sel])]


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_full_mix_verdicts_and_reach(precision):
    import bench
    g = np.load(os.path.join(GOLDEN, "ik_mix_reach.npz"))
    wl, pk, _ = _solve(precision)
    flags = bench.gpu_reach_flags(wl, [pk.q_of(i) for i in range(len(wl))])
    conv = ((pk.status & 0xFF) == 0).cpu().numpy()
    off = 0
    agree_all = []
    for ci, c in enumerate(wl):
        n = len(c["n_targets"])
        ref_reach = _per_class(g, ci, "reached").astype(bool)
        ref_conv = _per_class(g, ci, "converged").astype(bool)
        br_conv = _per_class(g, ci, "ref_converged").astype(bool)
        det = _per_class(g, ci, "margin") > MARGIN_ULPS
        assert len(ref_reach) == n
        mine = conv[off:off + n]
        agree = flags[ci] == ref_reach
        agree_all.append(agree)
        assert agree.mean() >= 0.98, (c["name"], agree.mean())
        a_det = (mine == ref_conv)[det].mean()
        # one line per class for the parity summary (shown with pytest -s)
        print(f"\n[parity] {precision} {c['name']}: n {n} determinate {int(det.sum())} "
              f"verdict(det) vs oracle {a_det:.4f} vs BetterRobot {(mine == br_conv)[det].mean():.4f} "
              f"verdict(rounding) vs oracle {(mine == ref_conv)[~det].mean():.4f} "
              f"(BetterRobot vs oracle {(br_conv == ref_conv)[~det].mean():.4f}) reach {agree.mean():.4f} "
              f"converged {int(mine.sum())}/{int(ref_conv.sum())}/{int(br_conv.sum())} (gpu/oracle/BetterRobot)")
        if precision == "f64":
            assert a_det >= 0.999, (c["name"], a_det)
            assert (mine == br_conv)[det].mean() >= 0.999, c["name"]
            br_round = (br_conv == ref_conv)[~det].mean()
            assert (mine == ref_conv)[~det].mean() >= br_round - 0.05, (c["name"], br_round)
        else:
            assert a_det >= (0.975 if c["name"] == "humanoid" else 0.99), (c["name"], a_det)
        off += n
    agree_all = np.concatenate(agree_all)
    assert agree_all.mean() >= 0.99, agree_all.mean()
    ours, ref = sum(int(f.sum()) for f in flags), int(g["reached"].sum())
    assert abs(ours - ref) <= 0.01 * ref, (ours, ref)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_full_mix_final_residuals(precision):
    """Where both converged, the stacked residual at the GPU's solution and at the oracle's final
    configuration (both evaluated by the kernel: 0 iterations from that configuration) agree
    within 1e-4 on >= 99% of problems."""
    from betterrobot_b200 import ik as bik
    g = np.load(os.path.join(GOLDEN, "ik_mix_reach.npz"))
    if "q_final" not in g.files:
        pytest.skip("fixture without final configurations")
    wl, pk, settings = _solve(precision)
    conv = ((pk.status & 0xFF) == 0).cpu().numpy()

    def residuals(qs):
        pr = bik.PackedIK([c["model"] for c in wl], [c["frames"] for c in wl], [c["n_targets"] for c in wl],
                          team_sizes=[32] * len(wl), warps_per_cta=4, with_residual=True)
        pr.set_inputs([c["targets"] for c in wl], qs)
        s0 = bik.IKSettings.from_buffer_copy(settings)
        s0.max_iter = 0
        pr.solve(s0)
        torch.cuda.synchronize()
        return pr
    mine = residuals([pk.q_of(i).clone() for i in range(len(wl))])
    qf, qo = g["q_final"], g["q_offset"]
    ref_q = []
    for ci, c in enumerate(wl):
        nq = c["model"].nq
        idx = np.nonzero(g["cls"] == ci)[0][np.argsort(g["index"][g["cls"] == ci])]
        ref_q.append(torch.from_numpy(np.stack([qf[qo[i]:qo[i] + nq] for i in idx])).float().cuda())
    ref = residuals(ref_q)
    rm, rr = mine.residual.cpu().numpy(), ref.residual.cpu().numpy()
    both = conv & _cat(g, "converged", wl).astype(bool)
    ok = []
    for p in np.nonzero(both)[0]:
        a, b = mine.r_offset_np[p], mine.r_offset_np[p] + mine.r_dim[p]
        ok.append(np.abs(rm[a:b] - rr[a:b]).max() <= 1e-4)
    assert np.mean(ok) >= 0.99, np.mean(ok)


def _cat(g, key, wl):
    return np.concatenate([_per_class(g, ci, key) for ci in range(len(wl))])

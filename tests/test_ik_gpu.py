"""GPU parity of the persistent LM / GN kernel against the reference solver (float64).

Bar (float32 kernel vs float64 reference/oracle):
* same converged / not-converged verdict;
* final stacked residual within 1e-4 (max abs difference of the residual vectors);
checked on the reference's own float64 solves (golden fixtures) and on larger
seeded batches against the oracle.  The kernel decides accept / reject and
convergence on a float64 cost; its float32 normal equations still move iterates
by ~1e-7, which can flip a verdict on problems that end right at the tolerance,
so the batch tests require the bar on >= 90-95% of problems (measured 94-100%).
"""

import os

import numpy as np
import pytest
import torch

from betterrobot_b200 import ik as bik, synthetic as syn
from oracle import ik as oik, kinematics as K

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

RES_TOL = 1e-4
SPECS = {"chain7": syn.chain_spec(), "humanoid": syn.humanoid_spec(), "dual_arm": syn.dual_arm_spec(),
         "mixed": syn.mixed_spec()}


def _models(name):
    return syn.model_from_spec(SPECS[name]), syn.model_from_spec(SPECS[name], dtype=torch.float64)


def _cfgs(st, optimizer="lm", g=None):
    cost = bik.IKCostConfig(limit_weight=float(st[4]), rest_weight=float(st[5]))
    opt = bik.OptimizerConfig(optimizer=optimizer, max_iter=int(st[3]), tol=float(st[2]),
                              lam0=float(st[0]) if st[0] else 1e-4, factor=float(st[1]) if st[1] else 2.0)
    if g is not None and "damping" in g:
        opt.damping = str(g["damping"])
        opt.gn_eps = float(g["gn_eps"])
    return cost, opt


def _oracle_margins(g, robot):
    """The oracle's decision margins on a golden case (the oracle reproduces these solves with the
    same iterations and verdicts, tests/test_oracle_golden.py)."""
    _, m64 = _models(robot)
    st = g["settings"]
    constant = "damping" in g and str(g["damping"]) == "constant"
    s = oik.IKSettings(lam0=st[0] or 1e-4, factor=1.0 if constant else (st[1] or 2.0), tol=st[2],
                       max_iter=int(st[3]), limit_weight=st[4], rest_weight=st[5], optimizer=str(g["optimizer"]),
                       kernel=str(g["kernel"]) if "kernel" in g else "l2")
    kinds = [str(k) for k in g["kinds"]] if "kinds" in g else None
    return oik.solve(m64, [int(f) for f in g["frame_ids"]], g["targets"], g["q0"], s, kinds=kinds).margin


def _agreement(out, ref_conv, ref_res):
    conv = out.converged.cpu().numpy()
    res = out.residual.cpu().double().numpy()
    dres = np.abs(res - ref_res).max(axis=1)
    ok = (conv == ref_conv) & (dres <= RES_TOL)
    return ok, conv, dres


@pytest.mark.parametrize("case,robot", [("chain7_random", "chain7"), ("chain7_gn", "chain7"),
                                        ("dual_arm", "dual_arm"), ("humanoid", "humanoid"),
                                        ("chain7_huber", "chain7"), ("chain7_gn_cauchy", "chain7"),
                                        ("dual_arm_cauchy", "dual_arm"), ("humanoid_tukey", "humanoid"),
                                        ("chain7_position", "chain7"), ("dual_arm_mixed", "dual_arm"),
                                        ("humanoid_mixed", "humanoid"), ("mixed", "mixed"),
                                        ("chain7_constant", "chain7")])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_reference_solver_golden(case, robot, precision):
    """The reference's own float64 solves (l2, the robust IRLS kernels, Constant damping)
    reproduced on the GPU.  With float64 normal equations every verdict that the float64 sum's
    rounding does not decide (oracle decision margin > 64 units of the cost's spacing) is the
    reference's, with the final residual within 1e-4."""
    g = np.load(os.path.join(GOLDEN, f"ik_{case}.npz"))
    m, _ = _models(robot)
    cost, opt = _cfgs(g["settings"], str(g["optimizer"]), g)
    opt.kernel = str(g["kernel"]) if "kernel" in g else "l2"
    opt.precision = precision
    fids = [int(f) for f in g["frame_ids"]]
    kinds = [str(k) for k in g["kinds"]] if "kinds" in g else None
    out = bik.solve_ik_batched(m, fids, torch.from_numpy(g["targets"]).float().cuda(),
                               torch.from_numpy(g["q0"]).float().cuda(), cost_cfg=cost, optimizer_cfg=opt,
                               with_residual=True, target_kinds=kinds)
    ok, conv, dres = _agreement(out, g["converged"], g["residual"])
    # every converged reference solve must converge here to the same residual
    both = g["converged"].astype(bool)
    assert (conv[both]).all(), (conv, g["converged"])
    assert (dres[both] <= RES_TOL).all(), dres
    assert ok.mean() >= 0.75, (ok, conv, g["converged"], dres)
    if precision == "f64":
        det = _oracle_margins(g, robot) > 64
        assert (conv == g["converged"])[det].all(), (conv, g["converged"], det)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_singular_normal_equations_take_the_minimum_norm_step(precision):
    """GN without damping (eps = 0) on the dual-arm with one left-arm target and no limit / rest
    terms: the right arm's Jacobian columns are zero, J^T J is exactly singular, and the kernel's
    factorization meets zero pivots.  Its retry with a 1e-6 diagonal gives the minimum-norm
    Gauss-Newton step (zero on the idle arm), as the oracle's least-squares fallback does:
    every problem converges, the idle arm does not move, and the final residual matches the
    oracle's within 1e-4.  The reference (golden) takes the lstsq branch of
    optim/solvers/cholesky.py:14-20 instead; on an exactly singular matrix its rank decision is
    made on rounding noise (torch's gelsy rank estimate), and none of these six solves converges
    there in 30 iterations (torch.linalg.lstsq on the oracle's own, mathematically equal H
    converges on two of them): that path is not reproducible and is not the bar here."""
    g = np.load(os.path.join(GOLDEN, "ik_dual_arm_gn_singular.npz"))
    m, m64 = _models("dual_arm")
    cost, opt = _cfgs(g["settings"], "gn", g)
    opt.precision = precision
    fids = [int(f) for f in g["frame_ids"]]
    out = bik.solve_ik_batched(m, fids, torch.from_numpy(g["targets"]).float().cuda(),
                               torch.from_numpy(g["q0"]).float().cuda(), cost_cfg=cost, optimizer_cfg=opt,
                               with_residual=True)
    s = oik.IKSettings(optimizer="gn", gn_eps=0.0, limit_weight=0.0, rest_weight=0.0, tol=float(g["settings"][2]),
                       max_iter=int(g["settings"][3]))
    ref = oik.solve(m64, fids, g["targets"], g["q0"], s)
    assert ref.converged.all() and not g["converged"].any()
    conv = out.converged.cpu().numpy()
    assert conv.all(), conv
    assert ((out.status.cpu().numpy() >> 8) & 2).all()         # BR_IK_FLAG_REGULARIZED: the retry ran
    q = out.q.cpu().double().numpy()
    idle = [int(m.idx_qs[j]) for j, name in enumerate(m.joint_names) if name.startswith("r") and m.nqs[j] == 1]
    assert idle and np.abs(q[:, idle] - g["q0"][:, idle]).max() <= 1e-6
    res = out.residual.cpu().double().numpy()
    assert np.abs(res - ref.residual).max() <= RES_TOL


def _config0(P, seed):
    m, m64 = _models("chain7")
    fid = m.frame_id("ee")
    q_goal = syn.random_q(m64, P, seed, rev_range=2.8)
    q0 = syn.random_q(m64, P, seed + 1, rev_range=2.8)
    oMi, _ = K.forward_kinematics(m64, q_goal.numpy())
    targets = K.frame_placements(m64, oMi, [fid])
    return m, m64, fid, targets, q0


def test_config0_chain_random_starts_vs_oracle():
    """Config 0: 256 chains, q0 and target-q uniform in the limits, LM 1e-3 x10, 50 iters, tol 1e-6."""
    m, m64, fid, targets, q0 = _config0(256, 40)
    s = oik.IKSettings(lam0=1e-3, factor=10.0, tol=1e-6, max_iter=50)
    ref = oik.solve(m64, [fid], targets, q0.numpy(), s)
    out = bik.solve_ik_batched(m, [fid], torch.from_numpy(targets).float().cuda(), q0.float().cuda(),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=50, lam0=1e-3, factor=10.0),
                               with_residual=True)
    ok, conv, dres = _agreement(out, ref.converged, ref.residual)
    both = ref.converged & conv
    assert (conv == ref.converged).mean() >= 0.95, (conv.mean(), ref.converged.mean())
    assert np.median(dres[both]) <= RES_TOL
    assert (dres[both] <= RES_TOL).mean() >= 0.95


@pytest.mark.parametrize("robot,frames,rest,P,agree_min", [
    ("chain7", ["ee"], 1e-3, 64, 0.9), ("dual_arm", ["ee_l", "ee_r"], 1e-3, 64, 0.9),
    ("humanoid", ["track0", "track1", "track2", "track3"], 1e-3, 64, 0.9),
    # mixed robot: planar base + translation lift are redundant; with a rest term the float64
    # LM converges on 9% of these problems in 100 iterations, without it on 73% (median 33)
    ("mixed", ["ee", "mid"], 0.0, 64, 0.9),
    ("humanoid", ["track0", "track4"], 0.01, 128, 0.85)])
def test_noisy_start_vs_oracle(robot, frames, rest, P, agree_min):
    """Config-3 style problems: targets from FK(q*), q0 = q* + N(0, 0.3), 100 iterations.

    Verdict agreement has a floor set by float32 itself.  On the humanoid two-target case
    with rest weight 0.01, the oracle's own LM run with a float32 Jacobian (normal
    equations formed in float32, or formed exactly and solved with one step of iterative
    refinement) agrees with the float64 run on 0.88-0.91 of these 128 problems: the
    disagreeing problems take different paths from the first iterations (one run converges
    in 35-60 iterations, the other is still going at 100), not near the iteration limit.
    That case therefore asks for 0.85, and for no bias in the converged rate.
    """
    m, m64 = _models(robot)
    fids = [m.frame_id(f) for f in frames]
    q_star = syn.random_q(m64, P, 50, rev_range=2.5, base_translation=0.5)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    targets = K.frame_placements(m64, oMi, fids)
    q0 = syn.noisy_start(m64, q_star, 0.3, 51)
    s = oik.IKSettings(lam0=1e-3, factor=10.0, tol=1e-6, max_iter=100, rest_weight=rest)
    ref = oik.solve(m64, fids, targets, q0.numpy(), s)
    out = bik.solve_ik_batched(m, fids, torch.from_numpy(targets).float().cuda(), q0.float().cuda(),
                               cost_cfg=bik.IKCostConfig(rest_weight=rest),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=100, lam0=1e-3, factor=10.0),
                               with_residual=True)
    ok, conv, dres = _agreement(out, ref.converged, ref.residual)
    # final residuals are compared where the float64 solve converged: elsewhere they record
    # where each run stopped at the iteration limit
    done = ref.converged.astype(bool)
    assert (dres[done] <= RES_TOL).mean() >= 0.95, (np.sort(dres[done])[-8:], done.mean())
    assert (conv == ref.converged).mean() >= agree_min, (conv.mean(), ref.converged.mean())
    assert abs(conv.mean() - ref.converged.mean()) <= 0.08, (conv.mean(), ref.converged.mean())


@pytest.mark.parametrize("spec", [syn.chain_spec(seed=9, n=62, name="chain62"),
                                  syn.floating_chain_spec(seed=9, n=58)], ids=["chain62", "floating58"])
def test_size_limit_trees_vs_oracle(spec):
    """Trees at the size limits: a 62-revolute chain (64 joints = BR_MAX_JOINTS) and a free-flyer
    with 58 revolutes (nv = 64 = BR_MAX_NV).  FK + frame Jacobian against the oracle, and 16
    noisy-start LM solves with the same verdicts and residuals."""
    m, m64 = syn.model_from_spec(spec), syn.model_from_spec(spec, dtype=torch.float64)
    fid = m.frame_id("ee")
    P = 16
    q_star = syn.random_q(m64, P, 70, rev_range=2.5, base_translation=1.0)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    targets = K.frame_placements(m64, oMi, [fid])
    import betterrobot_b200 as br
    T, J = br.frame_jacobians(m, q_star.float().cuda(), [fid])
    Jref = K.frame_jacobian(m64, oMi, q_star.numpy(), fid, "local_world_aligned")
    assert np.abs(T.cpu().double().numpy()[:, 0, :3] - targets[:, 0, :3]).max() <= 1e-4
    assert np.abs(J.cpu().double().numpy()[:, 0] - Jref).max() <= 1e-4 * np.abs(Jref).max()
    q0 = syn.noisy_start(m64, q_star, 0.3, 71)
    s = oik.IKSettings(lam0=1e-3, factor=10.0, tol=1e-6, max_iter=100, rest_weight=0.0)
    ref = oik.solve(m64, [fid], targets, q0.numpy(), s)
    assert ref.converged.all()
    out = bik.solve_ik_batched(m, [fid], torch.from_numpy(targets).float().cuda(), q0.float().cuda(),
                               cost_cfg=bik.IKCostConfig(rest_weight=0.0),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=100, lam0=1e-3, factor=10.0),
                               with_residual=True)
    ok, conv, dres = _agreement(out, ref.converged, ref.residual)
    assert ok.mean() >= 0.9, (conv.mean(), dres.max())


def test_inconsistent_tree_tables_are_refused():
    """A class whose tree under-reports its DOF entries, or whose level schedule holds an offset
    outside the factor storage, is refused problem by problem (status flag BADTREE, x = x0)
    by the kernel's own checks before any of it is used; the same batch then solves normally."""
    from betterrobot_b200.tree import TreeArrays
    m, m64 = _models("humanoid")
    fids = [m.frame_id(f) for f in ("track0", "track2")]
    P = 64
    q_star = syn.random_q(m64, P, 60, rev_range=2.5, base_translation=0.5)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    targets = torch.from_numpy(K.frame_placements(m64, oMi, fids)).float().cuda()
    q0 = syn.noisy_start(m64, q_star, 0.3, 61).float().cuda()
    frames = np.tile(np.array(fids, np.int32), (P, 1))
    pk = bik.PackedIK([m], [frames], [np.full(P, len(fids), np.int32)], team_sizes=[32], warps_per_cta=4)
    pk.set_inputs([targets], [q0])
    settings = bik.settings_from(bik.IKCostConfig(rest_weight=1e-3), bik.OptimizerConfig(max_iter=100))
    badtree = 4  # BR_IK_FLAG_BADTREE
    good_sched, good_ent = pk._trees[0].dof_sched, pk._trees[0].dof_entries

    sched = TreeArrays(m).dof_schedule().copy()
    toff = (5 + int(sched[0]) + 3) & ~3
    sched[toff] = (sched[toff] & np.uint32(0xffff0000)) | np.uint32(0xffff)   # first task's destination
    bad = torch.from_numpy(sched.view(np.int32)).cuda()
    for field, value in (("dof_sched", bad.data_ptr()), ("dof_entries", 10)):
        setattr(pk._trees[0], field, value)
        pk.solve(settings)
        st = pk.status.cpu().numpy()
        assert (((st >> 8) & badtree) != 0).all(), (field, st[:4])
        torch.testing.assert_close(pk.q_of(0), q0, rtol=0, atol=0)
        pk._trees[0].dof_sched, pk._trees[0].dof_entries = good_sched, good_ent
    pk.solve(settings)
    st = pk.status.cpu().numpy()
    assert (((st >> 8) & badtree) == 0).all()
    fresh = bik.PackedIK([m], [frames], [np.full(P, len(fids), np.int32)], team_sizes=[32], warps_per_cta=4)
    fresh.set_inputs([targets], [q0])
    fresh.solve(settings)
    np.testing.assert_array_equal(st, fresh.status.cpu().numpy())
    torch.testing.assert_close(pk.q_of(0), fresh.q_of(0), rtol=0, atol=0)


def test_uneven_mix_single_launch_matches_per_class():
    """Three robots, 1-6 targets, one launch == the same problems solved class by class."""
    models = [_models(n) for n in ("humanoid", "dual_arm", "chain7")]
    cand = {"humanoid": [f"track{i}" for i in range(6)], "dual_arm": ["ee_l", "ee_r", "body_l_link5",
            "body_r_link5", "body_l_link3", "body_r_link3"], "chain7": ["ee", "body_link7", "body_link6",
            "body_link5", "body_link4", "body_link3"]}
    rng = np.random.default_rng(3)
    frames, nts, tg, q0s = [], [], [], []
    for (m, m64), name in zip(models, ("humanoid", "dual_arm", "chain7")):
        P = 24
        fids = np.array([m.frame_id(f) for f in cand[name]], np.int32)
        nt = rng.integers(1, 7, size=P).astype(np.int32)
        q_star = syn.random_q(m64, P, 60, rev_range=2.5, base_translation=0.5)
        oMi, _ = K.forward_kinematics(m64, q_star.numpy())
        T = K.frame_placements(m64, oMi, list(fids))
        frames.append(np.broadcast_to(fids, (P, 6)))
        nts.append(nt)
        tg.append(torch.from_numpy(T).float())
        q0s.append(syn.noisy_start(m64, q_star, 0.3, 61).float())
    settings = bik.settings_from(bik.IKCostConfig(rest_weight=1e-3),
                                 bik.OptimizerConfig(max_iter=60, lam0=1e-3, factor=10.0))
    pk = bik.PackedIK([m for m, _ in models], frames, nts, with_residual=True)
    pk.set_inputs(tg, q0s)
    pk.solve(settings)
    for c, (m, m64) in enumerate(models):
        one = bik.PackedIK([m], [frames[c]], [nts[c]], with_residual=True)
        one.set_inputs([tg[c]], [q0s[c]])
        one.solve(settings)
        assert torch.equal(pk.q_of(c), one.q_of(0))
        assert torch.equal(pk.iters[pk.class_slice(c)], one.iters)


def test_solve_ik_single_problem_api():
    m, m64 = _models("dual_arm")
    q_star = syn.random_q(m64, 1, 70)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    fids = [m.frame_id("ee_l"), m.frame_id("ee_r")]
    T = K.frame_placements(m64, oMi, fids)[0]
    q0 = syn.noisy_start(m64, q_star, 0.2, 71)[0]
    res = bik.solve_ik(m, {"ee_l": torch.from_numpy(T[0]), "ee_r": torch.from_numpy(T[1])},
                       initial_q=q0.float().cuda(), cost_cfg=bik.IKCostConfig(rest_weight=1e-3),
                       optimizer_cfg=bik.OptimizerConfig(lam0=1e-3, factor=10.0))
    ref = oik.solve(m64, fids, T[None], q0.numpy()[None],
                    oik.IKSettings(lam0=1e-3, factor=10.0, max_iter=100, rest_weight=1e-3))
    assert res.q.shape == (m.nq,)
    assert res.residual.shape == (6 * 2 + 2 * m.nq + m.nv,)
    assert res.converged == bool(ref.converged[0])
    assert float((res.residual.cpu().double() - torch.from_numpy(ref.residual[0])).abs().max()) <= RES_TOL
    pose = res.frame_pose("ee_l").cpu().double().numpy()
    assert np.abs(pose[:3] - T[0, :3]).max() < 1e-3


def test_zero_iterations_returns_start_and_cost():
    m, m64 = _models("chain7")
    q0 = syn.random_q(m64, 5, 80)
    fid = m.frame_id("ee")
    T = torch.zeros(5, 1, 7)
    T[..., 6] = 1
    out = bik.solve_ik_batched(m, [fid], T.cuda(), q0.float().cuda(),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=0), with_residual=True)
    assert torch.equal(out.q.cpu(), q0.float())
    assert (out.iters == 0).all() and not out.converged.any()
    r, _ = oik.residual_and_jacobian(m64, q0.numpy(), [fid], T.double().numpy(), m64.q_neutral.numpy(),
                                     oik.IKSettings(), want_jac=False)
    np.testing.assert_allclose(out.residual.cpu().double().numpy(), r, atol=1e-5)
    np.testing.assert_allclose(out.cost.cpu().double().numpy(), 0.5 * (r * r).sum(-1), rtol=1e-5, atol=1e-6)


def test_unsupported_options_raise():
    m, _ = _models("chain7")
    T = torch.zeros(1, 1, 7, device="cuda")
    q0 = torch.zeros(1, m.nq, device="cuda")
    for opt in (bik.OptimizerConfig(optimizer="adam"), bik.OptimizerConfig(damping="trust_region"),
                bik.OptimizerConfig(linear_solver="lstsq")):
        with pytest.raises(NotImplementedError):
            bik.solve_ik_batched(m, [0], T, q0, optimizer_cfg=opt)
    with pytest.raises(bik.ShapeError):
        bik.solve_ik_batched(m, [m.nframes], T, q0)


def test_autotune_and_graph_replay_match_direct_solve():
    from betterrobot_b200 import autotune
    models = [_models(n) for n in ("humanoid", "chain7")]
    frames, nts, tg, q0s = [], [], [], []
    for (m, m64), names in zip(models, (["track0", "track1"], ["ee", "body_link5"])):
        P = 48
        fids = np.array([m.frame_id(f) for f in names], np.int32)
        q_star = syn.random_q(m64, P, 90, rev_range=2.5, base_translation=0.5)
        oMi, _ = K.forward_kinematics(m64, q_star.numpy())
        frames.append(np.broadcast_to(fids, (P, 2)))
        nts.append(np.full(P, 2, np.int32))
        tg.append(torch.from_numpy(K.frame_placements(m64, oMi, list(fids))).float().cuda())
        q0s.append(syn.noisy_start(m64, q_star, 0.3, 91).float().cuda())
    settings = bik.settings_from(bik.IKCostConfig(rest_weight=1e-3),
                                 bik.OptimizerConfig(max_iter=40, lam0=1e-3, factor=10.0))

    def make(teams, warps):
        p = bik.PackedIK([m for m, _ in models], frames, nts, team_sizes=teams, warps_per_cta=warps)
        p.set_inputs(tg, q0s)
        return p
    teams, warps, ms = autotune.tune(make, settings, reps=1)
    assert ms > 0 and len(teams) == 2
    ref = make(None, 4)
    ref.solve(settings)
    pk = make(teams, warps)
    g = pk.capture(settings)
    pk.x.fill_(float("nan"))
    g.replay()
    torch.cuda.synchronize()
    # team size changes the reduction order inside a problem: results agree to float32 rounding
    for c in range(2):
        assert float((pk.q_of(c) - ref.q_of(c)).abs().max()) < 1e-3
    assert (pk.status == ref.status).float().mean() >= 0.95


@pytest.mark.parametrize("kernel", ["huber", "cauchy", "tukey"])
def test_robust_kernels_vs_oracle(kernel):
    """IRLS-reweighted LM on noisy humanoid starts against the oracle's float64 IRLS LM.

    128 problems: verdict agreement sits at the float32 floor (~0.93 measured over the three
    kernels and l2), and with 64 problems one binomial standard deviation is 3 points."""
    m, m64 = _models("humanoid")
    P = 128
    fids = [m.frame_id(f) for f in ("track0", "track2", "track4")]
    q_star = syn.random_q(m64, P, 80, rev_range=2.5, base_translation=0.5)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    targets = K.frame_placements(m64, oMi, fids)
    q0 = syn.noisy_start(m64, q_star, 0.3, 81)
    s = oik.IKSettings(lam0=1e-3, factor=10.0, tol=1e-6, max_iter=100, rest_weight=1e-3, kernel=kernel)
    ref = oik.solve(m64, fids, targets, q0.numpy(), s)
    out = bik.solve_ik_batched(m, fids, torch.from_numpy(targets).float().cuda(), q0.float().cuda(),
                               cost_cfg=bik.IKCostConfig(rest_weight=1e-3),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=100, lam0=1e-3, factor=10.0, kernel=kernel),
                               with_residual=True)
    ok, conv, dres = _agreement(out, ref.converged, ref.residual)
    assert (dres <= RES_TOL).mean() >= 0.9, np.sort(dres)[-8:]
    assert (conv == ref.converged).mean() >= 0.85, (conv.mean(), ref.converged.mean())


@pytest.mark.parametrize("robot,frames,kinds", [
    ("chain7", ["ee"], ["position"]),
    ("dual_arm", ["ee_l", "ee_r"], ["position", "orientation"]),
    ("humanoid", ["track0", "track2", "track4"], ["pose", "position", "orientation"])])
def test_position_orientation_targets_vs_oracle(robot, frames, kinds):
    """PositionResidual / OrientationResidual targets (pose.py:107-195) against the float64 oracle."""
    m, m64 = _models(robot)
    P = 64
    fids = [m.frame_id(f) for f in frames]
    q_star = syn.random_q(m64, P, 90, rev_range=2.5, base_translation=0.5)
    oMi, _ = K.forward_kinematics(m64, q_star.numpy())
    targets = K.frame_placements(m64, oMi, fids)
    q0 = syn.noisy_start(m64, q_star, 0.3, 91)
    s = oik.IKSettings(lam0=1e-3, factor=10.0, tol=1e-6, max_iter=100, rest_weight=1e-3)
    ref = oik.solve(m64, fids, targets, q0.numpy(), s, kinds=kinds)
    out = bik.solve_ik_batched(m, fids, torch.from_numpy(targets).float().cuda(), q0.float().cuda(),
                               cost_cfg=bik.IKCostConfig(rest_weight=1e-3),
                               optimizer_cfg=bik.OptimizerConfig(max_iter=100, lam0=1e-3, factor=10.0),
                               with_residual=True, target_kinds=kinds)
    assert out.residual.shape == ref.residual.shape
    ok, conv, dres = _agreement(out, ref.converged, ref.residual)
    assert (dres <= RES_TOL).mean() >= 0.9, np.sort(dres)[-8:]
    assert (conv == ref.converged).mean() >= 0.85, (conv.mean(), ref.converged.mean())


def test_empty_problem_batch():
    """P = 0 problems: empty results, no launch."""
    m, _ = _models("chain7")
    out = bik.solve_ik_batched(m, [m.frame_id("ee")], torch.zeros(0, 1, 7, device="cuda"),
                               torch.zeros(0, m.nq, device="cuda"))
    assert out.q.shape == (0, m.nq)
    assert out.iters.shape == (0,) and out.converged.shape == (0,)
    out = bik.solve_ik_batched(m, [m.frame_id("ee")], torch.zeros(0, 1, 7, device="cuda"),
                               torch.zeros(0, m.nq, device="cuda"), with_residual=True)
    assert out.q.shape == (0, m.nq) and out.residual.numel() == 0

"""GPU parity of the batched trajectory optimiser (GN / LM) and its goal adjoint.

Bars:
* reference ``solve_trajopt`` (golden, float64): same converged verdict, trajectory
  within 1e-4 rad, final stacked residual within 1e-4;
* float64 oracle at the config-4 size (chain7, T = 64): same verdicts, trajectories
  within 1e-4, final cost within 1e-6 absolute + 1e-4 relative;
* goal-pose gradient (d cost / d eps, goal -> goal exp(eps)): against float64 central
  differences (eps 1e-6) of the goal term at the returned trajectory,
  |g - fd| <= 1e-4 |fd| + 2e-6 (the absolute part covers the float32 rounding of the
  returned trajectory, ~1e-7 rad per joint, which the kernel's float64 iterate does
  not have); against re-solved float64 optimal costs (envelope theorem), within
  2e-2 relative, for trajectories whose every solve converged.

Goals are start + U(+-0.5) rad per joint: with +-1 rad, undamped GN oscillates
without converging on ~20% of trajectories even in float64.
"""

import os

import numpy as np
import pytest
import torch

from betterrobot_b200 import synthetic as syn
from betterrobot_b200 import trajopt as btr
from oracle import kinematics as K, lie, trajopt as ot

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _setup(N, T, seed, spread=0.5):
    m, m64 = syn.model_from_spec(syn.chain_spec()), syn.model_from_spec(syn.chain_spec(), dtype=torch.float64)
    fid = m.frame_id("ee")
    qs, qg = syn.trajopt_endpoints(m64, N, seed, spread)
    oMi, _ = K.forward_kinematics(m64, qg.numpy())
    goal = K.frame_placements(m64, oMi, [fid])[:, 0]
    oMi, _ = K.forward_kinematics(m64, qs.numpy())
    start = K.frame_placements(m64, oMi, [fid])[:, 0]
    X0 = np.repeat(qs.numpy()[:, None, :], T, 1)
    return m, m64, fid, goal, start, X0


def _gpu(m, fid, goal, start, X0, cfg):
    return btr.solve_trajopt_batched(m, fid, torch.from_numpy(goal).float().cuda(),
                                     torch.from_numpy(X0).float().cuda(),
                                     start=torch.from_numpy(start).float().cuda(), cfg=cfg)


@pytest.mark.parametrize("fixture", ["trajopt_chain7.npz", "trajopt_floating.npz", "trajopt_mixed.npz",
                                     "trajopt_humanoid.npz"])
def test_reference_solve_trajopt_golden(fixture):
    """The reference's float64 solve_trajopt: the 7-DOF chain, a floating-base chain, the
    robot with planar, translation, spherical and unbounded-revolute joints (knots moved by
    Model.integrate, acceleration and reference residuals through Model.difference), and the
    36-DOF free-flyer humanoid (a 72 x 72 boundary system over four warps)."""
    g = np.load(os.path.join(GOLDEN, fixture))
    T, dt, wg, ws, wa, wl, wr, tol, mi = g["settings"]
    spec = {"trajopt_chain7.npz": syn.chain_spec(), "trajopt_floating.npz": syn.floating_chain_spec(),
            "trajopt_mixed.npz": syn.mixed_spec(), "trajopt_humanoid.npz": syn.humanoid_spec()}[fixture]
    m = syn.model_from_spec(spec)
    m64 = syn.model_from_spec(spec, dtype=torch.float64)
    fid = m.frame_id(str(g["frame"]) if "frame" in g else "ee")
    X0 = np.repeat(g["q_start"][:, None, :], int(T), 1)
    cfg = btr.TrajOptConfig(dt=float(dt), w_goal=float(wg), w_start=float(ws), w_accel=float(wa), w_limit=float(wl),
                            w_ref=float(wr), tol=float(tol), max_iter=int(mi))
    out = _gpu(m, fid, g["goal"], g["start"], X0, cfg)
    np.testing.assert_array_equal(out.converged.cpu().numpy(), g["converged"])
    X = out.q.cpu().double().numpy()
    assert np.abs(X - g["X"]).max() <= 1e-4, np.abs(X - g["X"]).max()
    s = ot.TrajSettings(dt=dt, w_goal=wg, w_start=ws, w_accel=wa, w_limit=wl, w_ref=wr, tol=tol, max_iter=int(mi))
    r, _ = ot.residual_jacobian(m64, X, fid, g["goal"], g["start"], X0, s, want_jac=False)
    assert np.abs(r - g["residual"]).max() <= 1e-4


@pytest.mark.parametrize("optimizer", ["gn", "lm"])
def test_config4_size_vs_oracle(optimizer):
    T, N = 64, 16
    m, m64, fid, goal, start, X0 = _setup(N, T, 51)
    cfg = btr.TrajOptConfig(optimizer=optimizer, max_iter=30)
    out = _gpu(m, fid, goal, start, X0, cfg)
    s = ot.TrajSettings(optimizer=optimizer, max_iter=30)
    ref = ot.solve(m64, X0, fid, goal, start, s)
    conv = out.converged.cpu().numpy()
    assert (conv == ref.converged).mean() >= 0.9, (conv, ref.converged)
    both = conv & ref.converged
    X = out.q.cpu().double().numpy()
    assert np.abs(X[both] - ref.X[both]).max() <= 1e-4
    cost = out.cost.cpu().double().numpy()
    np.testing.assert_allclose(cost[both], ref.cost[both], rtol=1e-4, atol=1e-6)


def test_goal_gradient_adjoint_vs_float64_fd():
    T, N = 64, 8
    m, m64, fid, goal, start, X0 = _setup(N, T, 61)
    cfg = btr.TrajOptConfig(max_iter=30)
    s = ot.TrajSettings(max_iter=30)
    out = _gpu(m, fid, goal, start, X0, cfg)
    X = out.q.cpu().double().numpy()
    g = out.goal_grad.cpu().double().numpy()
    goal32 = goal.astype(np.float32).astype(np.float64)
    h = 1e-6
    fd = np.zeros((N, 6))
    for k in range(6):
        e = np.zeros((N, 6))
        e[:, k] = h
        gp = lie.se3_compose(goal32, lie.se3_exp(e))
        gm = lie.se3_compose(goal32, lie.se3_exp(-e))
        fd[:, k] = (ot.goal_cost(m64, X, fid, gp, s) - ot.goal_cost(m64, X, fid, gm, s)) / (2 * h)
    err = np.linalg.norm(g - fd, axis=1)
    assert (err <= 1e-4 * np.linalg.norm(fd, axis=1) + 2e-6).all(), (err, np.linalg.norm(fd, axis=1))


def test_goal_gradient_envelope_vs_resolved_cost():
    """d(optimal cost)/d(goal) by re-solving in float64 equals the adjoint at convergence."""
    T, N = 64, 4
    m, m64, fid, goal, start, X0 = _setup(N, T, 71)
    cfg = btr.TrajOptConfig(max_iter=60, tol=1e-8)
    s = ot.TrajSettings(max_iter=60, tol=1e-10)
    out = _gpu(m, fid, goal, start, X0, cfg)
    g = out.goal_grad.cpu().double().numpy()
    ok = out.converged.cpu().numpy().copy()
    h = 1e-5
    fd = np.zeros((N, 6))
    for k in range(6):
        e = np.zeros((N, 6))
        e[:, k] = h
        rp = ot.solve(m64, X0, fid, lie.se3_compose(goal, lie.se3_exp(e)), start, s)
        rm = ot.solve(m64, X0, fid, lie.se3_compose(goal, lie.se3_exp(-e)), start, s)
        ok &= rp.converged & rm.converged
        fd[:, k] = (rp.cost - rm.cost) / (2 * h)
    assert ok.sum() >= 2, ok
    rel = np.linalg.norm(g - fd, axis=1) / np.maximum(np.linalg.norm(fd, axis=1), 1e-12)
    assert (rel[ok] <= 2e-2).all(), rel


def _vs_oracle(spec, N, T, seed, frame="ee", spread=0.5):
    """N trajectories of T knots on ``spec`` against the float64 oracle (same verdicts on >= 90%,
    trajectories within 1e-4 and costs within 1e-6 + 1e-4 relative where both converged)."""
    m, m64 = syn.model_from_spec(spec), syn.model_from_spec(spec, dtype=torch.float64)
    fid = m.frame_id(frame)
    qs, qg = syn.trajopt_endpoints(m64, N, seed, spread)
    oMi, _ = K.forward_kinematics(m64, qg.numpy())
    goal = K.frame_placements(m64, oMi, [fid])[:, 0]
    oMi, _ = K.forward_kinematics(m64, qs.numpy())
    start = K.frame_placements(m64, oMi, [fid])[:, 0]
    X0 = np.repeat(qs.numpy()[:, None, :], T, 1)
    out = _gpu(m, fid, goal, start, X0, btr.TrajOptConfig(max_iter=30))
    # the oracle starts from the float32-rounded inputs the kernel saw
    X0r = X0.astype(np.float32).astype(np.float64)
    ref = ot.solve(m64, X0r, fid, goal.astype(np.float32).astype(np.float64),
                   start.astype(np.float32).astype(np.float64), ot.TrajSettings(max_iter=30))
    conv = out.converged.cpu().numpy()
    assert (conv == ref.converged).mean() >= 0.9, (conv, ref.converged)
    both = conv & ref.converged
    assert both.any()
    X = out.q.cpu().double().numpy()
    assert np.abs(X[both] - ref.X[both]).max() <= 1e-4, np.abs(X[both] - ref.X[both]).max()
    c = out.cost.cpu().double().numpy()
    assert (np.abs(c[both] - ref.cost[both]) <= 1e-6 + 1e-4 * np.abs(ref.cost[both])).all()


def test_floating_base_vs_oracle():
    """Floating-base chain (free-flyer knots), 16 trajectories x 24 knots, against the float64 oracle."""
    _vs_oracle(syn.floating_chain_spec(), 16, 24, 47)


def test_humanoid_vs_oracle():
    """The 36-DOF free-flyer humanoid (the FK + Jacobian robot), 6 trajectories x 16 knots
    (576 variables each), against the float64 oracle."""
    _vs_oracle(syn.humanoid_spec(), 6, 16, 57, frame="track0", spread=0.3)


@pytest.mark.parametrize("spec,N,T", [(syn.chain_spec(seed=11, n=16, name="chain16"), 16, 16),
                                      (syn.chain_spec(seed=13, n=62, name="chain62"), 3, 12),
                                      (syn.chain_spec(), 8, 128)], ids=["nv16", "nv62", "knots128"])
def test_size_limits_vs_oracle(spec, N, T):
    """The trajectory limits: nv = 16 (a 32 x 32 boundary system: one warp's substitutions),
    nv = 62 (64 joints, the tree table's limit: a 124 x 124 boundary system over the whole
    CTA) and T = 128 = BR_MAX_TRAJ_KNOTS knots."""
    _vs_oracle(spec, N, T, 53)


@pytest.mark.parametrize("T", [3, 9, 10, 11])
def test_band_factorization_paths_vs_oracle(T):
    """Around the switch to the twisted band factorization (>= 8 interior knots: T >= 10): the
    one-ended path at T = 3 and 9, the smallest twisted cases at T = 10 (2 bottom rows) and
    T = 11 (an odd band), against the float64 oracle."""
    _vs_oracle(syn.chain_spec(), 12, T, 59)


def test_trajopt_rejects_oversized_trees_and_bad_shapes():
    m = syn.model_from_spec(syn.humanoid_spec())     # 128 knots of 36 DOFs: above shared memory
    X0 = torch.zeros(2, 128, m.nq, device="cuda")
    X0[..., 6] = 1.0
    with pytest.raises(Exception):
        btr.solve_trajopt_batched(m, m.frame_id("track0"), torch.zeros(2, 7, device="cuda"), X0)
    mc = syn.model_from_spec(syn.chain_spec())
    with pytest.raises(btr.ShapeError):
        btr.solve_trajopt_batched(mc, 0, torch.zeros(3, 7, device="cuda"), torch.zeros(2, 8, mc.nq, device="cuda"))


class _Item:
    def __init__(self, residual, weight):
        self.residual, self.weight, self.active = residual, weight, True


class _Stack:
    """The shape of BetterRobot's CostStack that solve_trajopt reads (``items``: name -> item)."""

    def __init__(self):
        self.items = {}

    def add(self, name, residual, weight=1.0):
        self.items[name] = _Item(residual, weight)


def _ref_like(name, **attrs):
    """An object whose class is named like a BetterRobot residual / optimizer, with its attributes."""
    return type(name, (), {})() if not attrs else type(name, (), dict(attrs))()


def test_solve_trajopt_facade_matches_reference_golden():
    """``solve_trajopt(model, horizon=, dt=, initial_q_traj=, cost_stack=, optimizer=)`` with the
    stack the reference's golden solves used (objects shaped like BetterRobot's, the reference
    itself not being importable here) returns the reference's trajectories."""
    g = np.load(os.path.join(GOLDEN, "trajopt_chain7.npz"))
    T, dt, wg, ws, wa, wl, wr, tol, mi = g["settings"]
    T = int(T)
    m = syn.model_from_spec(syn.chain_spec())
    fid = m.frame_id("ee")
    for n in range(len(g["X"])):
        X0 = torch.from_numpy(np.repeat(g["q_start"][n][None], T, 0))
        st = _Stack()
        pose = lambda target: _ref_like("PoseResidual", frame_id=fid, target=torch.from_numpy(target),  # noqa: E731
                                        pos_weight=1.0, ori_weight=1.0)
        st.add("goal", _ref_like("TimeIndexedResidual", inner=pose(g["goal"][n]), t_idx=T - 1), float(wg))
        st.add("start", _ref_like("TimeIndexedResidual", inner=pose(g["start"][n]), t_idx=0), float(ws))
        st.add("accel", _ref_like("AccelerationResidual", dt=float(dt), weight=1.0), float(wa))
        for t in range(T):
            st.add(f"limits_t{t}", _ref_like("TimeIndexedResidual", inner=_ref_like("JointPositionLimit", weight=1.0),
                                             t_idx=t), float(wl))
        st.add("ref", _ref_like("ReferenceTrajectoryResidual", q_ref=X0.clone(), weight=1.0), float(wr))
        r = btr.solve_trajopt(m, horizon=T, dt=float(dt), initial_q_traj=X0.cuda(), cost_stack=st,
                              optimizer=_ref_like("GaussNewton", tol=float(tol), eps=1e-8), max_iter=int(mi))
        assert r.converged == bool(g["converged"][n])
        assert r.trajectory.q.shape == (1, T, m.nq)
        assert np.abs(r.trajectory.q[0].cpu().double().numpy() - g["X"][n]).max() <= 1e-4
    with pytest.raises(NotImplementedError):
        st.add("other", _ref_like("CollisionResidual"), 1.0)
        btr.solve_trajopt(m, horizon=T, dt=float(dt), initial_q_traj=X0.cuda(), cost_stack=st,
                          optimizer=_ref_like("GaussNewton", tol=1e-6, eps=1e-8))


def test_empty_trajectory_batch():
    """N = 0 trajectories: empty results, no launch."""
    m = syn.model_from_spec(syn.chain_spec())
    out = btr.solve_trajopt_batched(m, m.frame_id("ee"), torch.zeros(0, 7, device="cuda"),
                                    torch.zeros(0, 16, m.nq, device="cuda"))
    assert out.q.shape == (0, 16, m.nq)
    assert out.converged.shape == (0,) and out.iters.shape == (0,)

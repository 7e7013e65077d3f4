"""Generate the golden fixtures that pin the oracle to BetterRobot itself.

Run where the reference source tree is available (it is read, never copied):

    python tests/golden/make_golden.py /path/to/BetterRobot/src

For each synthetic robot (``betterrobot_b200.synthetic``) the script builds the
reference ``Model`` with the reference's own ``ModelBuilder`` + ``build_model``
in float64, runs the reference's torch code on seeded inputs and stores inputs
and outputs in ``tests/golden/*.npz``:

* ``lie.npz``       — ``se3_exp/log``, ``so3_exp/log`` (incl. theta -> 0 and qw < 0),
                      ``right_jacobian_inv_se3`` (the truncated-series inverse).
* ``lie_ops.npz``   — every other LieOps method (compose, inverse, act, adjoint(_inv),
                      normalize, to/from matrix) and ``right_jacobian_se3``.
* ``kin_<robot>.npz`` — ``forward_kinematics`` (oMi, liMi), ``frame_pose_world``,
                      ``get_frame_jacobian`` in all three reference frames,
                      ``compute_joint_jacobians``, plus the reference model's topology
                      arrays so tests can check the local ``Model`` builds the same tree.
* ``ik_<case>.npz`` — float64 LM / GN solves built exactly as ``solve_ik`` builds them
                      (``tasks/ik.py:191-226``) but with the configs' damping.
* ``adjoint.npz``   — pose loss ``sum_f w_f |log(T_f^-1 oMf(q))|^2`` and its autograd
                      gradient w.r.t. raw ``q`` (free-flyer quaternion included).
* ``trajopt_floating.npz``, ``trajopt_mixed.npz`` — the same ``solve_trajopt`` stack on a
                      floating-base chain and on the robot with every multi-slot joint kind
                      (acceleration and reference residuals through ``Model.difference``).
* ``adjoint_mixed.npz`` — the same on the robot with every multi-slot joint kind
                      (planar, translation, spherical, unbounded revolute).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from betterrobot_b200 import synthetic as syn  # noqa: E402

D = torch.float64


def reference_model(spec):
    from better_robot.io.build_model import build_model
    from better_robot.io.parsers.programmatic import ModelBuilder

    b = ModelBuilder(spec["name"])
    joints = spec["joints"]
    bodies = {0: "universe"}
    for i, rec in enumerate(joints):
        bodies[i + 1] = rec["body"]
        b.add_body(rec["body"])
    for i, rec in enumerate(joints):
        origin = torch.tensor(rec.get("origin", [0, 0, 0, 0, 0, 0, 1.0]), dtype=D)
        if i == 0:
            if rec["kind"] == "free_flyer":
                b.add_free_flyer_root(rec["name"], child=rec["body"], origin=origin)
            continue  # fixed root: build_model inserts "root_joint" itself
        parent_body = bodies[rec["parent"]]
        kw = dict(parent=parent_body, child=rec["body"], origin=origin)
        if rec["kind"] == "revolute_rz":
            b.add_revolute_z(rec["name"], lower=rec["lower"], upper=rec["upper"], **kw)
        elif rec["kind"] == "revolute_ry":
            b.add_revolute_y(rec["name"], lower=rec["lower"], upper=rec["upper"], **kw)
        elif rec["kind"] == "revolute_unbounded":
            b.add_revolute(rec["name"], axis=torch.tensor(rec["axis"], dtype=D), unbounded=True, **kw)
        elif rec["kind"] == "spherical":
            b.add_spherical(rec["name"], **kw)
        elif rec["kind"] == "planar":
            b.add_planar(rec["name"], **kw)
        elif rec["kind"] == "translation":
            from better_robot.data_model.joint_models.translation import JointTranslation
            b.add_joint(rec["name"], kind=JointTranslation(), **kw)
        else:
            raise NotImplementedError(rec["kind"])
    for fr in spec["frames"]:
        b.add_frame(fr["name"], parent_body=bodies[fr["parent"]],
                    placement=torch.tensor(fr["placement"], dtype=D))
    return build_model(b.finalize(), dtype=D)


def topology_arrays(m):
    return {
        "parents": np.array(m.parents), "nqs": np.array(m.nqs), "nvs": np.array(m.nvs),
        "idx_qs": np.array(m.idx_qs), "idx_vs": np.array(m.idx_vs),
        "kinds": np.array([jm.kind for jm in m.joint_models]),
        "joint_placements": m.joint_placements.numpy(),
        "lower": m.lower_pos_limit.numpy(), "upper": m.upper_pos_limit.numpy(),
        "frame_parent": np.array([f.parent_joint for f in m.frames]),
        "frame_placement": torch.stack([f.joint_placement for f in m.frames]).numpy(),
        "frame_names": np.array(m.frame_names), "q_neutral": m.q_neutral.numpy(),
    }


def make_lie(out):
    from better_robot.lie import _torch_native_backend as tn
    from better_robot.lie.tangents import right_jacobian_inv_se3

    g = torch.Generator().manual_seed(11)
    xi = torch.randn(64, 6, generator=g, dtype=D)
    xi[:, 3:] *= torch.linspace(0.0, 3.0, 64, dtype=D)[:, None] / xi[:, 3:].norm(dim=-1, keepdim=True)
    xi[0, 3:] = 0.0
    xi[1, 3:] = 1e-5
    xi[2, 3:] = torch.tensor([3e-5, -2e-5, 1e-5], dtype=D)
    T = tn.se3_exp(xi)
    Tq = T.clone()
    Tq[::3, 3:] = -Tq[::3, 3:]  # double cover: qw < 0 rows
    np.savez_compressed(out, xi=xi.numpy(), se3_exp=T.numpy(), T_in=Tq.numpy(), se3_log=tn.se3_log(Tq).numpy(),
                        so3_exp=tn.so3_exp(xi[:, 3:]).numpy(), so3_log=tn.so3_log(Tq[:, 3:]).numpy(),
                        jr_inv=right_jacobian_inv_se3(xi).numpy())


def make_lie_ops(out):
    """The remaining LieOps methods and ``right_jacobian_se3``, with rotations that take each
    branch of ``_matrix_to_quat`` (trace > 0, then m00 / m11 / m22 largest) and angles near pi."""
    from better_robot.lie import _torch_native_backend as tn
    from better_robot.lie.tangents import right_jacobian_se3

    g = torch.Generator().manual_seed(12)
    n = 64
    q = torch.randn(n, 4, generator=g, dtype=D)
    q = q / q.norm(dim=-1, keepdim=True)
    # near-pi rotations about x, y, z (qw ~ 0, both signs) and one exactly at pi
    for i, ax in enumerate((0, 1, 2, 0, 1, 2)):
        q[i] = 0.0
        q[i, ax] = 1.0
        q[i, 3] = (1e-4 if i < 3 else -1e-4)
        q[i] = q[i] / q[i].norm()
    q[6] = torch.tensor([0.0, 0.0, 1.0, 0.0], dtype=D)
    q[7] = torch.tensor([0.0, 0.0, 0.0, 1.0], dtype=D)
    t = torch.randn(n, 3, generator=g, dtype=D)
    A = torch.cat([t, q], -1)
    qb = torch.randn(n, 4, generator=g, dtype=D)
    qb = qb / qb.norm(dim=-1, keepdim=True)
    B = torch.cat([torch.randn(n, 3, generator=g, dtype=D), qb], -1)
    P = torch.randn(n, 3, generator=g, dtype=D)
    scale = torch.rand(n, 1, generator=g, dtype=D) * 1.5 + 0.25
    A_unnorm = torch.cat([t, q * scale], -1)
    xi = torch.randn(n, 6, generator=g, dtype=D)
    xi[:, 3:] *= torch.linspace(0.0, 3.0, n, dtype=D)[:, None] / xi[:, 3:].norm(dim=-1, keepdim=True)
    xi[0, 3:] = 0.0
    R = tn.so3_to_matrix(q)
    np.savez_compressed(
        out, A=A.numpy(), B=B.numpy(), P=P.numpy(), A_unnorm=A_unnorm.numpy(), xi=xi.numpy(),
        se3_compose=tn.se3_compose(A, B).numpy(), se3_inverse=tn.se3_inverse(A).numpy(),
        se3_act=tn.se3_act(A, P).numpy(), se3_adjoint=tn.se3_adjoint(A).numpy(),
        se3_adjoint_inv=tn.se3_adjoint_inv(A).numpy(), se3_normalize=tn.se3_normalize(A_unnorm).numpy(),
        se3_log=tn.se3_log(A).numpy(), so3_log=tn.so3_log(q).numpy(),
        so3_compose=tn.so3_compose(q, qb).numpy(), so3_inverse=tn.so3_inverse(q).numpy(),
        so3_act=tn.so3_act(q, P).numpy(), so3_to_matrix=R.numpy(), so3_from_matrix=tn.so3_from_matrix(R).numpy(),
        so3_normalize=tn.so3_normalize(q * scale).numpy(), jr=right_jacobian_se3(xi).numpy())


def make_kin(name, spec, batch, seed, base_t, out):
    from better_robot.kinematics.forward import forward_kinematics
    from better_robot.kinematics.jacobian import compute_joint_jacobians, get_frame_jacobian

    m = reference_model(spec)
    mine = syn.model_from_spec(spec, dtype=D)
    q = syn.random_q(mine, batch, seed, rev_range=2.5, base_translation=base_t)
    data = forward_kinematics(m, q, compute_frames=True)
    ops = [i for i, f in enumerate(m.frames) if f.frame_type != "body"]
    sel = ops + [m.njoints - 1]
    Js = {}
    for ref in ("world", "local_world_aligned", "local"):
        Js[ref] = torch.stack([get_frame_jacobian(m, data, f, reference=ref) for f in sel], -3).numpy()
    data2 = forward_kinematics(m, q)
    compute_joint_jacobians(m, data2)
    # Model.integrate / Model.difference (data_model/model.py:160-190) on the same configurations
    v = torch.from_numpy(np.random.default_rng(seed + 50).normal(0.0, 0.4, size=(batch, m.nv)))
    q1 = syn.noisy_start(mine, q, 0.3, seed + 51)
    np.savez_compressed(out, q=q.numpy(), oMi=data.joint_pose_world.numpy(), liMi=data.joint_pose_local.numpy(),
                        v=v.numpy(), q1=q1.numpy(), integrate=m.integrate(q, v).numpy(),
                        difference=m.difference(q, q1).numpy(),
                        oMf=data.frame_pose_world.numpy(), frame_ids=np.array(sel),
                        J_world=Js["world"], J_lwa=Js["local_world_aligned"], J_local=Js["local"],
                        joint_jacobians=data2.joint_jacobians.numpy(), **topology_arrays(m))


def reference_lm(m, frame_names, targets, q0, *, tol, max_iter, lam0=1e-3, factor=10.0, pos_w=1.0, ori_w=1.0,
                 limit_w=0.1, rest_w=0.01, optimizer="lm", kernel="l2", kinds=None, damping="adaptive",
                 gn_eps=1e-8):
    """One float64 solve through the reference's own stack (``tasks/ik.py:191-258``)."""
    from better_robot.costs.stack import CostStack
    from better_robot.kinematics.forward import forward_kinematics
    from better_robot.optim.optimizers.gauss_newton import GaussNewton
    from better_robot.optim.optimizers.levenberg_marquardt import LevenbergMarquardt
    from better_robot.optim.problem import LeastSquaresProblem
    from better_robot.optim.solvers.cholesky import Cholesky
    from better_robot.optim.strategies.adaptive import Adaptive
    from better_robot.optim.strategies.constant import Constant
    from better_robot.residuals.base import ResidualState
    from better_robot.residuals.limits import JointPositionLimit
    from better_robot.residuals.pose import PoseResidual
    from better_robot.residuals.regularization import RestResidual

    from better_robot.residuals.pose import OrientationResidual, PositionResidual

    stack = CostStack()
    for i, (name, T) in enumerate(zip(frame_names, targets)):
        kind = "pose" if kinds is None else kinds[i]
        if kind == "position":
            res = PositionResidual(frame_id=m.frame_id(name), target=T, weight=pos_w)
        elif kind == "orientation":
            res = OrientationResidual(frame_id=m.frame_id(name), target=T, weight=ori_w)
        else:
            res = PoseResidual(frame_id=m.frame_id(name), target=T, pos_weight=pos_w, ori_weight=ori_w)
        stack.add(f"{kind}_{name}", res, weight=1.0)
    if limit_w > 0:
        stack.add("limits", JointPositionLimit(m), weight=limit_w)
    if rest_w > 0:
        stack.add("rest", RestResidual(m, m.q_neutral), weight=rest_w)

    def sf(x):
        return ResidualState(model=m, data=forward_kinematics(m, x, compute_frames=True), variables=x)

    prob = LeastSquaresProblem(cost_stack=stack, state_factory=sf, x0=q0.clone(), lower=m.lower_pos_limit,
                               upper=m.upper_pos_limit, nv=m.nv, retract=lambda q, dv: m.integrate(q, dv))
    from better_robot.tasks.ik import _make_robust_kernel
    k = _make_robust_kernel(kernel)   # solve_ik's own factory: None for "l2"
    if optimizer == "lm":
        # solve_ik's OptimizerConfig.damping (tasks/ik.py:136-147): Adaptive, or Constant (lambda fixed)
        strat = Constant(lam=lam0) if damping == "constant" else Adaptive(lam0=lam0, factor=factor)
        st = LevenbergMarquardt(lam0=lam0, factor=factor, tol=tol).minimize(
            prob, max_iter=max_iter, linear_solver=Cholesky(), kernel=k, strategy=strat)
    else:
        st = GaussNewton(tol=tol, eps=gn_eps).minimize(prob, max_iter=max_iter, linear_solver=Cholesky(), kernel=k)
    return st


def make_ik(case, spec, frame_names, P, seed, start, out, **kw):
    m = reference_model(spec)
    mine = syn.model_from_spec(spec, dtype=D)
    from better_robot.kinematics.forward import forward_kinematics
    q_star = syn.random_q(mine, P, seed, rev_range=2.5, base_translation=0.5)
    if start == "random":
        q0 = syn.random_q(mine, P, seed + 100, rev_range=2.8)
    else:
        q0 = syn.noisy_start(mine, q_star, 0.3, seed + 200)
    data = forward_kinematics(m, q_star, compute_frames=True)
    fids = [m.frame_id(n) for n in frame_names]
    targets = data.frame_pose_world[:, fids, :].clone()
    res = {"q": [], "iters": [], "converged": [], "residual": [], "cost": []}
    for p in range(P):
        st = reference_lm(m, frame_names, targets[p], q0[p], **kw)
        res["q"].append(st.x.numpy())
        res["iters"].append(st.iters)
        res["converged"].append(st.status == "converged")
        res["residual"].append(st.residual.numpy())
        res["cost"].append(float(st.residual_norm))
    np.savez_compressed(out, q_star=q_star.numpy(), q0=q0.numpy(), targets=targets.numpy(),
                        frame_ids=np.array(fids), q_final=np.stack(res["q"]), iters=np.array(res["iters"]),
                        converged=np.array(res["converged"]), residual=np.stack(res["residual"]),
                        cost=np.array(res["cost"]),
                        settings=np.array([kw.get("lam0", 0), kw.get("factor", 0), kw["tol"], kw["max_iter"],
                                           kw.get("limit_w", 0.1), kw.get("rest_w", 0.01)]),
                        optimizer=np.array(kw.get("optimizer", "lm")), kernel=np.array(kw.get("kernel", "l2")),
                        kinds=np.array(kw.get("kinds") or ["pose"] * len(frame_names)),
                        damping=np.array(kw.get("damping", "adaptive")), gn_eps=np.array(kw.get("gn_eps", 1e-8)))


def make_ik_kernels(chain, dual, hum, lm):
    """Robust-kernel (IRLS) solves: random starts put chain residual rows outside Huber's
    quadratic region; Cauchy and Tukey reweight every row."""
    make_ik("chain7_huber", chain, ["ee"], 8, 25, "random", os.path.join(HERE, "ik_chain7_huber.npz"),
            max_iter=50, kernel="huber", **lm)
    make_ik("chain7_gn_cauchy", chain, ["ee"], 6, 26, "noisy", os.path.join(HERE, "ik_chain7_gn_cauchy.npz"),
            max_iter=30, tol=1e-6, optimizer="gn", kernel="cauchy")
    make_ik("dual_arm_cauchy", dual, ["ee_l", "ee_r"], 4, 27, "noisy", os.path.join(HERE, "ik_dual_arm_cauchy.npz"),
            max_iter=100, rest_w=1e-3, kernel="cauchy", **lm)
    make_ik("humanoid_tukey", hum, ["track0", "track2", "track4"], 4, 28, "noisy",
            os.path.join(HERE, "ik_humanoid_tukey.npz"), max_iter=100, rest_w=1e-3, kernel="tukey", **lm)


def make_ik_mixed():
    """LM on the robot with every multi-slot joint kind.  Most of its noisy-start solves run
    the full 100 iterations without converging, and where such a run ends depends on the
    float rounding of every step, so 24 problems (not 6) to measure agreement on."""
    make_ik("mixed", syn.mixed_spec(), ["ee", "mid"], 24, 32, "noisy", os.path.join(HERE, "ik_mixed.npz"),
            max_iter=100, rest_w=1e-3, lam0=1e-3, factor=10.0, tol=1e-6)


def make_ik_kinds(chain, dual, hum, lm):
    """Stacks with PositionResidual / OrientationResidual targets (residuals/pose.py:107-195)."""
    make_ik("chain7_position", chain, ["ee"], 8, 29, "noisy", os.path.join(HERE, "ik_chain7_position.npz"),
            max_iter=50, kinds=["position"], **lm)
    make_ik("dual_arm_mixed", dual, ["ee_l", "ee_r"], 4, 30, "noisy", os.path.join(HERE, "ik_dual_arm_mixed.npz"),
            max_iter=100, rest_w=1e-3, kinds=["position", "orientation"], **lm)
    make_ik("humanoid_mixed", hum, ["track0", "track2", "track4"], 4, 31, "noisy",
            os.path.join(HERE, "ik_humanoid_mixed.npz"), max_iter=100, rest_w=1e-3,
            kinds=["pose", "position", "orientation"], **lm)


def make_ik_damping_and_singular(chain, dual):
    """LM with Constant damping (solve_ik's damping="constant": Constant() keeps lambda = 1e-4,
    optim/strategies/constant.py:9-25); and GN without damping (eps = 0) on the dual-arm with one
    left-arm target and no limit / rest terms: the right arm's Jacobian columns are zero, so
    J^T J is exactly singular, torch.linalg.cholesky fails and Cholesky.solve falls back to
    lstsq (optim/solvers/cholesky.py:14-20) in every iteration."""
    make_ik("chain7_constant", chain, ["ee"], 8, 33, "noisy", os.path.join(HERE, "ik_chain7_constant.npz"),
            max_iter=60, tol=1e-6, lam0=1e-4, factor=2.0, damping="constant")
    make_ik("dual_arm_gn_singular", dual, ["ee_l"], 6, 34, "noisy", os.path.join(HERE, "ik_dual_arm_gn_singular.npz"),
            max_iter=30, tol=1e-6, optimizer="gn", gn_eps=0.0, limit_w=0.0, rest_w=0.0)


def make_adjoint(spec, B, seed, out):
    from better_robot.kinematics.forward import forward_kinematics
    from better_robot.lie import se3

    m = reference_model(spec)
    mine = syn.model_from_spec(spec, dtype=D)
    q = syn.random_q(mine, B, seed, rev_range=2.5, base_translation=1.0)
    ops = [i for i, f in enumerate(m.frames) if f.frame_type != "body"]
    targets = syn.random_targets(B, len(ops), seed + 1)
    rng = np.random.default_rng(seed + 2)
    w = torch.from_numpy(rng.uniform(0.5, 2.0, size=len(ops)))
    qv = q.clone().requires_grad_(True)
    data = forward_kinematics(m, qv, compute_frames=True)
    oMf = data.frame_pose_world[:, ops, :]
    xi = se3.log(se3.compose(se3.inverse(targets), oMf))
    loss = ((xi * xi).sum(-1) * w).sum(-1)
    (g,) = torch.autograd.grad(loss.sum(), qv)
    np.savez_compressed(out, q=q.numpy(), targets=targets.numpy(), weights=w.numpy(), frame_ids=np.array(ops),
                        loss=loss.detach().numpy(), grad=g.numpy())


def make_trajopt(spec, N, T, seed, out, dt=0.05, w_goal=1.0, w_start=1.0, w_accel=1e-2, w_limit=0.1,
                 w_ref=1e-3, tol=1e-6, max_iter=30, spread=1.0, frame="ee"):
    """Reference solve_trajopt (knots, GaussNewton) on the config-4 stack, float64."""
    from better_robot.costs.stack import CostStack
    from better_robot.kinematics.forward import forward_kinematics
    from better_robot.optim.optimizers.gauss_newton import GaussNewton
    from better_robot.residuals import AccelerationResidual, JointPositionLimit, PoseResidual, TimeIndexedResidual
    from better_robot.residuals.regularization import ReferenceTrajectoryResidual
    from better_robot.tasks.trajopt import solve_trajopt

    m = reference_model(spec)
    mine = syn.model_from_spec(spec, dtype=D)
    q_start, q_goal = syn.trajopt_endpoints(mine, N, seed, spread)
    fid = m.frame_id(frame)
    res = {"X": [], "iters": [], "converged": [], "residual": []}
    goals, starts = [], []
    for n in range(N):
        Tg = forward_kinematics(m, q_goal[n], compute_frames=True).frame_pose_world[fid].clone()
        Ts = forward_kinematics(m, q_start[n], compute_frames=True).frame_pose_world[fid].clone()
        X0 = q_start[n].expand(T, -1).clone()
        stack = CostStack()
        stack.add("goal", TimeIndexedResidual(PoseResidual(frame_id=fid, target=Tg), t_idx=T - 1), weight=w_goal)
        stack.add("start", TimeIndexedResidual(PoseResidual(frame_id=fid, target=Ts), t_idx=0), weight=w_start)
        stack.add("accel", AccelerationResidual(m, dt=dt), weight=w_accel)
        for t in range(T):
            stack.add(f"limits_t{t}", TimeIndexedResidual(JointPositionLimit(m), t_idx=t, name=f"limits_t{t}"),
                      weight=w_limit)
        stack.add("ref", ReferenceTrajectoryResidual(m, X0.clone()), weight=w_ref)
        r = solve_trajopt(m, horizon=T, dt=dt, initial_q_traj=X0, cost_stack=stack, optimizer=GaussNewton(tol=tol),
                          max_iter=max_iter)
        res["X"].append(r.trajectory.q[0].numpy())
        res["iters"].append(r.iters)
        res["converged"].append(r.converged)
        res["residual"].append(r.residual.numpy())
        goals.append(Tg.numpy())
        starts.append(Ts.numpy())
    np.savez_compressed(out, q_start=q_start.numpy(), q_goal=q_goal.numpy(), goal=np.stack(goals),
                        start=np.stack(starts), X=np.stack(res["X"]), iters=np.array(res["iters"]),
                        converged=np.array(res["converged"]), residual=np.stack(res["residual"]),
                        settings=np.array([T, dt, w_goal, w_start, w_accel, w_limit, w_ref, tol, max_iter]),
                        frame=np.array(frame))


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else None
    if src:
        sys.path.insert(0, src)
    torch.set_default_dtype(D)
    only = sys.argv[2:]
    if only == ["adjoint_mixed"]:   # regenerate one fixture: make_golden.py <src> adjoint_mixed
        make_adjoint(syn.mixed_spec(), 8, 33, os.path.join(HERE, "adjoint_mixed.npz"))
        return
    if only == ["trajopt_floating"]:
        make_trajopt(syn.floating_chain_spec(), 3, 12, 43, os.path.join(HERE, "trajopt_floating.npz"))
        return
    if only == ["ik_mixed"]:
        make_ik_mixed()
        return
    if only == ["trajopt_mixed"]:
        make_trajopt(syn.mixed_spec(), 3, 12, 45, os.path.join(HERE, "trajopt_mixed.npz"), spread=0.3)
        return
    if only == ["ik_damping"]:
        make_ik_damping_and_singular(syn.chain_spec(), syn.dual_arm_spec())
        return
    if only == ["trajopt_humanoid"]:
        make_trajopt(syn.humanoid_spec(), 2, 10, 49, os.path.join(HERE, "trajopt_humanoid.npz"), spread=0.3,
                     frame="track0")
        return
    make_lie(os.path.join(HERE, "lie.npz"))
    make_lie_ops(os.path.join(HERE, "lie_ops.npz"))
    chain, hum, dual = syn.chain_spec(), syn.humanoid_spec(), syn.dual_arm_spec()
    make_kin("chain7", chain, 16, 5, 0.0, os.path.join(HERE, "kin_chain7.npz"))
    make_kin("humanoid", hum, 8, 6, 1.0, os.path.join(HERE, "kin_humanoid.npz"))
    make_kin("dual_arm", dual, 8, 7, 0.0, os.path.join(HERE, "kin_dual_arm.npz"))
    make_kin("mixed", syn.mixed_spec(), 16, 8, 0.0, os.path.join(HERE, "kin_mixed.npz"))
    lm = dict(lam0=1e-3, factor=10.0, tol=1e-6)
    make_ik("chain7_random", chain, ["ee"], 8, 21, "random", os.path.join(HERE, "ik_chain7_random.npz"),
            max_iter=50, **lm)
    make_ik("chain7_noisy_gn", chain, ["ee"], 6, 22, "noisy", os.path.join(HERE, "ik_chain7_gn.npz"),
            max_iter=30, tol=1e-6, optimizer="gn")
    make_ik("dual_arm", dual, ["ee_l", "ee_r"], 4, 23, "noisy", os.path.join(HERE, "ik_dual_arm.npz"),
            max_iter=100, rest_w=1e-3, **lm)
    make_ik("humanoid", hum, ["track0", "track2", "track4"], 4, 24, "noisy",
            os.path.join(HERE, "ik_humanoid.npz"), max_iter=100, rest_w=1e-3, **lm)
    make_ik_kernels(chain, dual, hum, lm)
    make_ik_kinds(chain, dual, hum, lm)
    make_ik_mixed()
    make_ik_damping_and_singular(chain, dual)
    make_adjoint(hum, 4, 31, os.path.join(HERE, "adjoint.npz"))
    make_adjoint(syn.mixed_spec(), 8, 33, os.path.join(HERE, "adjoint_mixed.npz"))
    make_trajopt(chain, 3, 24, 41, os.path.join(HERE, "trajopt_chain7.npz"))
    make_trajopt(syn.floating_chain_spec(), 3, 12, 43, os.path.join(HERE, "trajopt_floating.npz"))
    make_trajopt(syn.mixed_spec(), 3, 12, 45, os.path.join(HERE, "trajopt_mixed.npz"), spread=0.3)
    make_trajopt(syn.humanoid_spec(), 2, 10, 49, os.path.join(HERE, "trajopt_humanoid.npz"), spread=0.3,
                 frame="track0")


if __name__ == "__main__":
    main()

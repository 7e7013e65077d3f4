"""The float64 oracle reproduces BetterRobot's own outputs (golden fixtures made by the reference)."""

import os

import numpy as np
import pytest
import torch

from betterrobot_b200 import synthetic as syn
from oracle import ik, kinematics as K, lie

from conftest import GOLDEN

SPECS = {"chain7": syn.chain_spec(), "humanoid": syn.humanoid_spec(), "dual_arm": syn.dual_arm_spec(),
         "mixed": syn.mixed_spec()}


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.mark.parametrize("robot", list(SPECS))
def test_local_model_matches_reference_tree(robot):
    g = _load(f"kin_{robot}.npz")
    m = syn.model_from_spec(SPECS[robot], dtype=torch.float64)
    assert tuple(g["parents"]) == m.parents
    assert list(g["kinds"]) == [jm.kind for jm in m.joint_models]
    np.testing.assert_array_equal(g["idx_qs"], m.idx_qs)
    np.testing.assert_array_equal(g["idx_vs"], m.idx_vs)
    np.testing.assert_array_equal(g["joint_placements"], m.joint_placements.numpy())
    np.testing.assert_array_equal(g["lower"], m.lower_pos_limit.numpy())
    np.testing.assert_array_equal(g["upper"], m.upper_pos_limit.numpy())
    assert list(g["frame_names"]) == list(m.frame_names)
    np.testing.assert_array_equal(g["frame_parent"], [f.parent_joint for f in m.frames])
    np.testing.assert_allclose(g["frame_placement"], torch.stack([f.joint_placement for f in m.frames]).numpy(),
                               atol=0, rtol=0)
    np.testing.assert_array_equal(g["q_neutral"], m.q_neutral.numpy())


@pytest.mark.parametrize("robot", list(SPECS))
def test_fk_frames_jacobians_match_reference(robot):
    g = _load(f"kin_{robot}.npz")
    m = syn.model_from_spec(SPECS[robot], dtype=torch.float64)
    oMi, liMi = K.forward_kinematics(m, g["q"])
    np.testing.assert_allclose(oMi, g["oMi"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(liMi, g["liMi"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(K.frame_placements(m, oMi), g["oMf"], atol=1e-12, rtol=0)
    for ref, key in (("world", "J_world"), ("local_world_aligned", "J_lwa"), ("local", "J_local")):
        J = np.stack([K.frame_jacobian(m, oMi, g["q"], int(f), ref) for f in g["frame_ids"]], -3)
        np.testing.assert_allclose(J, g[key], atol=1e-12, rtol=0)
    np.testing.assert_allclose(K.compute_joint_jacobians(m, oMi, g["q"]), g["joint_jacobians"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(K.integrate(m, g["q"], g["v"]), g["integrate"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(K.difference(m, g["q"], g["q1"]), g["difference"], atol=1e-12, rtol=0)


def test_lie_matches_reference():
    g = _load("lie.npz")
    np.testing.assert_allclose(lie.se3_exp(g["xi"]), g["se3_exp"], atol=1e-13, rtol=0)
    np.testing.assert_allclose(lie.se3_log(g["T_in"]), g["se3_log"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(lie.so3_exp(g["xi"][:, 3:]), g["so3_exp"], atol=1e-13, rtol=0)
    np.testing.assert_allclose(lie.so3_log(g["T_in"][:, 3:]), g["so3_log"], atol=1e-13, rtol=0)
    np.testing.assert_allclose(lie.right_jacobian_inv_se3(g["xi"]), g["jr_inv"], atol=1e-12, rtol=0)


@pytest.mark.parametrize("case,robot", [("chain7_random", "chain7"), ("chain7_gn", "chain7"),
                                        ("dual_arm", "dual_arm"), ("humanoid", "humanoid"),
                                        ("chain7_huber", "chain7"), ("chain7_gn_cauchy", "chain7"),
                                        ("dual_arm_cauchy", "dual_arm"), ("humanoid_tukey", "humanoid"),
                                        ("chain7_position", "chain7"), ("dual_arm_mixed", "dual_arm"),
                                        ("humanoid_mixed", "humanoid"), ("mixed", "mixed"),
                                        ("chain7_constant", "chain7")])
def test_lm_gn_match_reference_solver(case, robot):
    """The oracle's LM / GN reproduces the reference's solves; Constant damping
    (optim/strategies/constant.py:9-25) is Adaptive's update with factor 1."""
    g = _load(f"ik_{case}.npz")
    m = syn.model_from_spec(SPECS[robot], dtype=torch.float64)
    st = g["settings"]
    constant = "damping" in g and str(g["damping"]) == "constant"
    s = ik.IKSettings(lam0=st[0], factor=1.0 if constant else st[1], tol=st[2], max_iter=int(st[3]), limit_weight=st[4],
                      rest_weight=st[5], optimizer=str(g["optimizer"]),
                      kernel=str(g["kernel"]) if "kernel" in g else "l2")
    kinds = [str(k) for k in g["kinds"]] if "kinds" in g else None
    out = ik.solve(m, [int(f) for f in g["frame_ids"]], g["targets"], g["q0"], s, kinds=kinds)
    np.testing.assert_array_equal(out.iters, g["iters"])
    np.testing.assert_array_equal(out.converged, g["converged"])
    np.testing.assert_allclose(out.q, g["q_final"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(out.cost, g["cost"], atol=1e-12, rtol=1e-9)


def test_pose_loss_matches_reference():
    g = _load("adjoint.npz")
    m = syn.model_from_spec(SPECS["humanoid"], dtype=torch.float64)
    oMi, _ = K.forward_kinematics(m, g["q"])
    oMf = K.frame_placements(m, oMi, [int(f) for f in g["frame_ids"]])
    xi = lie.se3_log(lie.se3_compose(lie.se3_inverse(g["targets"]), oMf))
    loss = ((xi * xi).sum(-1) * g["weights"]).sum(-1)
    np.testing.assert_allclose(loss, g["loss"], atol=1e-12, rtol=1e-12)


def test_pose_loss_and_gradient_mixed_kinds_match_reference():
    """Loss and (float64 central-difference) gradient on the robot with every multi-slot
    joint kind against the reference's loss and autograd gradient."""
    g = _load("adjoint_mixed.npz")
    m = syn.model_from_spec(syn.mixed_spec(), dtype=torch.float64)
    fids = [int(f) for f in g["frame_ids"]]

    def loss_of(q):
        oMi, _ = K.forward_kinematics(m, q)
        oMf = K.frame_placements(m, oMi, fids)
        xi = lie.se3_log(lie.se3_compose(lie.se3_inverse(g["targets"]), oMf))
        return ((xi * xi).sum(-1) * g["weights"]).sum(-1)

    np.testing.assert_allclose(loss_of(g["q"]), g["loss"], atol=1e-12, rtol=1e-12)
    eps = 1e-6
    fd = np.zeros_like(g["q"])
    for i in range(g["q"].shape[1]):
        qp, qm = g["q"].copy(), g["q"].copy()
        qp[:, i] += eps
        qm[:, i] -= eps
        fd[:, i] = (loss_of(qp) - loss_of(qm)) / (2 * eps)
    np.testing.assert_allclose(fd, g["grad"], atol=1e-6 * np.abs(g["grad"]).max(), rtol=0)


def test_known_answers_one_joint_arm():
    """Reference known answers on a 1-joint arm (``tests/kinematics/test_fk.py:85-103``)."""
    import math
    m = syn.build_model("arm", [
        {"name": "root_joint", "kind": "fixed", "parent": 0, "body": "base"},
        {"name": "j1", "kind": "revolute_rz", "parent": 1, "body": "link1",
         "origin": [0, 0, 0.1, 0, 0, 0, 1], "lower": -math.pi, "upper": math.pi}], dtype=torch.float64)
    oMi, _ = K.forward_kinematics(m, np.zeros(1))
    assert abs(oMi[2, 2] - 0.1) < 1e-12
    oMi, _ = K.forward_kinematics(m, np.array([math.pi / 2]))
    assert abs(oMi[2, 5] - math.sin(math.pi / 4)) < 1e-12 and abs(oMi[2, 6] - math.cos(math.pi / 4)) < 1e-12


@pytest.mark.parametrize("fixture,spec", [("trajopt_chain7.npz", "chain7"), ("trajopt_floating.npz", "floating"),
                                          ("trajopt_mixed.npz", "mixed"), ("trajopt_humanoid.npz", "humanoid")])
def test_trajopt_matches_reference_solve_trajopt(fixture, spec):
    """GN trajectory optimisation (goal/start pose, acceleration, per-knot limits, reference
    trajectory), on the fixed-base chain, a floating-base chain (free-flyer knots), the
    robot with planar, translation, spherical and unbounded-revolute joints and the 36-DOF
    humanoid."""
    from oracle import trajopt as ot
    g = _load(fixture)
    T, dt, wg, ws, wa, wl, wr, tol, mi = g["settings"]
    m = syn.model_from_spec({"chain7": SPECS["chain7"], "floating": syn.floating_chain_spec(),
                             "mixed": syn.mixed_spec(), "humanoid": syn.humanoid_spec()}[spec], dtype=torch.float64)
    s = ot.TrajSettings(dt=dt, w_goal=wg, w_start=ws, w_accel=wa, w_limit=wl, w_ref=wr, tol=tol, max_iter=int(mi))
    X0 = np.repeat(g["q_start"][:, None, :], int(T), 1)
    fid = m.frame_id(str(g["frame"]) if "frame" in g else "ee")
    out = ot.solve(m, X0, fid, g["goal"], g["start"], s)
    np.testing.assert_array_equal(out.iters, g["iters"])
    np.testing.assert_array_equal(out.converged, g["converged"])
    np.testing.assert_allclose(out.X, g["X"], atol=1e-8, rtol=0)
    r, _ = ot.residual_jacobian(m, out.X, fid, g["goal"], g["start"], X0, s, want_jac=False)
    np.testing.assert_allclose(r, g["residual"], atol=1e-9, rtol=0)


def test_lie_ops_match_reference():
    """Every LieOps method and ``right_jacobian_se3`` (incl. rotations near pi and all Shepperd branches)."""
    g = _load("lie_ops.npz")
    A, B, P = g["A"], g["B"], g["P"]
    q, qb = A[:, 3:], B[:, 3:]
    checks = {
        "se3_compose": lie.se3_compose(A, B), "se3_inverse": lie.se3_inverse(A), "se3_act": lie.se3_act(A, P),
        "se3_adjoint": lie.se3_adjoint(A), "se3_adjoint_inv": lie.se3_adjoint_inv(A),
        "se3_normalize": lie.se3_normalize(g["A_unnorm"]), "se3_log": lie.se3_log(A), "so3_log": lie.so3_log(q),
        "so3_compose": lie.quat_mul(q, qb), "so3_inverse": lie.so3_inverse(q), "so3_act": lie.so3_act(q, P),
        "so3_to_matrix": lie.quat_to_matrix(q), "so3_from_matrix": lie.so3_from_matrix(g["so3_to_matrix"]),
        "so3_normalize": lie.so3_normalize(g["A_unnorm"][:, 3:]), "jr": lie.right_jacobian_se3(g["xi"]),
    }
    for k, v in checks.items():
        np.testing.assert_allclose(v, g[k], atol=1e-12, rtol=0, err_msg=k)


@pytest.mark.parametrize("fixture,spec", [("adjoint.npz", syn.humanoid_spec()), ("adjoint_mixed.npz", syn.mixed_spec())],
                         ids=["humanoid", "mixed"])
def test_oracle_pose_loss_gradient_matches_reference_autograd(fixture, spec):
    """The oracle's reverse sweep (oracle/adjoint.py) against BetterRobot's float64 autograd
    through its own FK (the humanoid, and the robot with every multi-slot joint kind)."""
    from oracle import adjoint as A
    g = np.load(os.path.join(GOLDEN, fixture))
    m64 = syn.model_from_spec(spec, dtype=torch.float64)
    L = A.pose_loss(m64, g["q"], g["frame_ids"], g["targets"], g["weights"])
    G = A.pose_loss_grad(m64, g["q"], g["frame_ids"], g["targets"], g["weights"])
    np.testing.assert_allclose(L, g["loss"], rtol=1e-12, atol=1e-12)
    assert np.abs(G - g["grad"]).max() <= 1e-12 * np.abs(g["grad"]).max()

"""Batched trajectory optimisation in float64 numpy — oracle only.

Restates ``solve_trajopt`` (``src/better_robot/tasks/trajopt.py:84-230``) with the
knot parameterisation and ``GaussNewton`` (``optim/optimizers/gauss_newton.py:27-76``)
or ``LevenbergMarquardt`` (``levenberg_marquardt.py:61-135``) on the cost stack

* ``goal``:  ``TimeIndexedResidual(PoseResidual(frame, T_goal), t = T-1)`` (``residuals/temporal.py:20-126``),
* ``start``: ``TimeIndexedResidual(PoseResidual(frame, T_start), t = 0)`` (optional),
* ``accel``: ``AccelerationResidual(model, dt)`` (``residuals/smoothness.py:98-161``),
* ``limits_t``: ``TimeIndexedResidual(JointPositionLimit(model), t)`` for every knot,
* ``ref``:   ``ReferenceTrajectoryResidual(model, q_ref)`` (``residuals/regularization.py:66-152``),

each with a scalar ``CostStack`` item weight (``costs/stack.py:104-144``), with the
dense ``(dim, T*nv)`` Jacobian the reference builds: the acceleration and reference
residuals through ``Model.difference`` with identity Jacobian blocks (the reference's
identity-right-Jacobian approximation, ``smoothness.py:98-108``), the limits through the
``(nq, nv)`` projection of ``limits.py:36-48`` (zero rows for joints with ``nq != nv``),
and the knot retraction through ``Model.integrate`` (``trajopt.py:159-169``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import ik as oik
from . import kinematics as K
from . import lie


@dataclass
class TrajSettings:
    dt: float = 0.05
    w_goal: float = 1.0
    w_start: float = 1.0
    w_accel: float = 1e-2
    w_limit: float = 0.1
    w_ref: float = 1e-3
    optimizer: str = "gn"
    tol: float = 1e-6
    max_iter: int = 30
    gn_eps: float = 1e-8
    lam0: float = 1e-3
    factor: float = 10.0


def _pose_rows(model, q, frame_id, target, want_jac):
    """PoseResidual value (6,) per trajectory and its analytic J (6, nv) at one knot (pose.py:58-103)."""
    oMi, _ = K.forward_kinematics(model, q)
    fr = model.frames[frame_id]
    Tee = lie.se3_compose(oMi[:, fr.parent_joint], K._np(fr.joint_placement))
    xi = lie.se3_log(lie.se3_compose(lie.se3_inverse(target), Tee))
    if not want_jac:
        return xi, None
    Jlwa = K.frame_jacobian(model, oMi, q, frame_id, "local_world_aligned")
    RT = np.swapaxes(lie.quat_to_matrix(Tee[:, 3:7]), -1, -2)
    Jloc = np.concatenate([RT @ Jlwa[:, :3], RT @ Jlwa[:, 3:]], -2)
    return xi, lie.right_jacobian_inv_se3(xi) @ Jloc


def residual_jacobian(model, X, frame_id, goal, start, q_ref, s: TrajSettings, want_jac=True):
    """Stacked residual (N, dim) and Jacobian (N, dim, T*nv) for trajectories X (N, T, nq)."""
    N, T, nq = X.shape
    nv = model.nv
    rs, Js = [], []

    def pose_block(t, target, w):
        xi, J = _pose_rows(model, X[:, t], frame_id, target, want_jac)
        rs.append(xi * w)
        if want_jac:
            full = np.zeros((N, 6, T * nv))
            full[:, :, t * nv:(t + 1) * nv] = J * w
            Js.append(full)

    if s.w_goal > 0:
        pose_block(T - 1, goal, s.w_goal)
    if s.w_start > 0 and start is not None:
        pose_block(0, start, s.w_start)
    if s.w_accel > 0:                                                   # smoothness.py:118-142
        c = s.w_accel / s.dt ** 2
        d = np.stack([K.difference(model, X[:, t], X[:, t + 1]) for t in range(T - 1)], 1)  # (N, T-1, nv)
        a = d[:, 1:] - d[:, :-1]
        rs.append((a * c).reshape(N, -1))
        if want_jac:
            J = np.zeros((N, (T - 2) * nv, T * nv))
            eye = np.eye(nv) * c
            for k in range(T - 2):
                J[:, k * nv:(k + 1) * nv, k * nv:(k + 1) * nv] = eye
                J[:, k * nv:(k + 1) * nv, (k + 1) * nv:(k + 2) * nv] = -2 * eye
                J[:, k * nv:(k + 1) * nv, (k + 2) * nv:(k + 3) * nv] = eye
            Js.append(J)
    if s.w_limit > 0:                                                   # limits.py:56-86 per knot
        lo = K._np(model.lower_pos_limit)
        hi = K._np(model.upper_pos_limit)
        dq_dv = np.zeros((nq, nv))                                      # limits.py:36-48
        for j, jm in enumerate(model.joint_models):
            if jm.nq and jm.nq == jm.nv:
                for k in range(jm.nq):
                    dq_dv[model.idx_qs[j] + k, model.idx_vs[j] + k] = 1.0
        for t in range(T):
            q = X[:, t]
            rs.append(np.concatenate([np.maximum(lo - q, 0.0), np.maximum(q - hi, 0.0)], -1) * s.w_limit)
            if want_jac:
                full = np.zeros((N, 2 * nq, T * nv))
                ld = np.where(q < lo, -1.0, 0.0)
                ud = np.where(q > hi, 1.0, 0.0)
                full[:, :nq, t * nv:(t + 1) * nv] = ld[..., None] * dq_dv * s.w_limit
                full[:, nq:, t * nv:(t + 1) * nv] = ud[..., None] * dq_dv * s.w_limit
                Js.append(full)
    if s.w_ref > 0:                                                     # regularization.py:133-152
        r_ref = np.stack([K.difference(model, q_ref[:, t], X[:, t]) for t in range(T)], 1)
        rs.append((r_ref * s.w_ref).reshape(N, -1))
        if want_jac:
            Js.append(np.broadcast_to(np.eye(T * nv) * s.w_ref, (N, T * nv, T * nv)))
    r = np.concatenate(rs, -1)
    return r, (np.concatenate(Js, -2) if want_jac else None)


@dataclass
class TrajOutcome:
    X: np.ndarray
    cost: np.ndarray
    iters: np.ndarray
    converged: np.ndarray


def solve(model, X0, frame_id, goal, start, s: TrajSettings, q_ref=None) -> TrajOutcome:
    """GN (or LM) on N independent trajectories, each following the single-problem reference loop."""
    X = np.array(X0, dtype=np.float64, copy=True)
    N, T, nq = X.shape
    q_ref = X.copy() if q_ref is None else np.asarray(q_ref, np.float64)
    ls = oik.IKSettings(lam0=s.lam0, factor=s.factor, tol=s.tol, max_iter=s.max_iter,
                        optimizer=s.optimizer, gn_eps=s.gn_eps)
    r, _ = residual_jacobian(model, X, frame_id, goal, start, q_ref, s, want_jac=False)
    cost = 0.5 * (r * r).sum(-1)
    lam = np.full(N, s.lam0)
    active = np.ones(N, bool)
    iters = np.full(N, s.max_iter)
    conv = np.zeros(N, bool)
    n = T * model.nv
    for it in range(s.max_iter):
        idx = np.nonzero(active)[0]
        if idx.size == 0:
            break
        r_a, J = residual_jacobian(model, X[idx], frame_id, goal[idx],
                                   None if start is None else start[idx], q_ref[idx], s)
        JtJ = np.swapaxes(J, -1, -2) @ J
        g = (np.swapaxes(J, -1, -2) @ r_a[..., None])[..., 0]
        damp = lam[idx] if s.optimizer == "lm" else np.full(idx.size, s.gn_eps)
        d = oik._solve(JtJ + damp[:, None, None] * np.eye(n), -g)
        d = d.reshape(-1, T, model.nv)                                   # knot retraction (trajopt.py:159-169)
        Xn = np.stack([K.integrate(model, X[idx][:, t], d[:, t]) for t in range(T)], 1)
        rn, _ = residual_jacobian(model, Xn, frame_id, goal[idx], None if start is None else start[idx],
                                  q_ref[idx], s, want_jac=False)
        cn = 0.5 * (rn * rn).sum(-1)
        gn = np.linalg.norm(g, axis=-1)
        if s.optimizer == "lm":
            acc = cn < cost[idx]
            X[idx[acc]] = Xn[acc]
            cost[idx[acc]] = cn[acc]
            lam[idx[acc]] = np.maximum(lam[idx[acc]] / s.factor, 1e-10)
            lam[idx[~acc]] = np.minimum(lam[idx[~acc]] * s.factor, 1e8)
            done = acc & (gn < s.tol)
        else:
            X[idx] = Xn
            cost[idx] = cn
            done = gn < s.tol
        conv[idx[done]] = True
        iters[idx[done]] = it + 1
        active[idx[done]] = False
    return TrajOutcome(X=X, cost=cost, iters=iters, converged=conv)


def goal_cost(model, X, frame_id, goal, s: TrajSettings) -> np.ndarray:
    """The goal-pose term of the cost, 0.5 |w_goal log(T_goal^-1 T_ee(q_{T-1}))|^2, per trajectory."""
    xi, _ = _pose_rows(model, X[:, -1], frame_id, goal, False)
    return 0.5 * (s.w_goal ** 2) * (xi * xi).sum(-1)


def total_cost(model, X, frame_id, goal, start, q_ref, s: TrajSettings) -> np.ndarray:
    r, _ = residual_jacobian(model, X, frame_id, goal, start, q_ref, s, want_jac=False)
    return 0.5 * (r * r).sum(-1)

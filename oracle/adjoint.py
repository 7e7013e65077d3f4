"""Pose loss through forward kinematics and its gradient w.r.t. raw q, float64 — oracle only.

The reference differentiates ``L(q) = sum_f w_f |log(T_f^-1 oMf(q))|^2`` by torch autograd
through its forward kinematics (``src/better_robot/kinematics/forward.py:73-135``, whose
list/stack design keeps the tape on purpose, ``forward.py:79-81``) and the SE3 ops of
``lie/_torch_native_backend.py``.  This restates that derivative as one reverse sweep:

* ``g_f = 2 w_f Jr^-1(xi_f)^T xi_f``: dL/d(right perturbation of oMf), with the exact SE3
  Jr^-1 (autograd differentiates ``se3_log`` exactly; the 40-term series of
  ``lie.right_jacobian_se3`` is exact to float64 for |xi| < 2 pi);
* ``F_f = Ad(oMf^-1)^T g_f``: the same sensitivity as a wrench at the world origin;
* ``dL/dv_c = sum_f <S_c, F_f>`` over the tangent columns that move frame f, with
  ``S_c = Ad(oMi_j) S_j`` the world twist of column c (``kinematics._joint_world_columns``);
* raw q of each joint kind: revolute / prismatic / translation ``dq = dv``; free-flyer
  ``t`` through R and the quaternion through its normalisation
  (``free_flyer.py:31-36``: ``delta_ang = 2 vec(u* (x) du)``, ``du = (I - u u^T) dq / |q|``);
  spherical likewise (``spherical.py:22-32``); unbounded revolute through
  ``th = atan2(s, c)`` (``revolute.py:206-211``); planar ``[x, y]`` through R and the angle
  through the half-angle formula of ``planar.py:20-41`` (``dth/dc = -1 / sin th``).

Pinned to the reference's own autograd gradients (``tests/golden/adjoint*.npz``) by
``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import numpy as np

from . import kinematics as K
from . import lie


def pose_loss(model, q, frame_ids, targets, weights) -> np.ndarray:
    """``(B,)`` loss for ``q (B, nq)``, ``targets (B, nf, 7)``, ``weights (nf,)`` or ``(B, nf)``."""
    oMi, _ = K.forward_kinematics(model, q)
    T = K.frame_placements(model, oMi, list(frame_ids))
    xi = lie.se3_log(lie.se3_compose(lie.se3_inverse(targets), T))
    return np.sum(np.asarray(weights) * np.sum(xi * xi, -1), -1)


def pose_loss_grad(model, q, frame_ids, targets, weights) -> np.ndarray:
    """``(B, nq)`` gradient of ``pose_loss`` w.r.t. raw ``q``."""
    q = K._np(q)
    B = q.shape[0]
    oMi, _ = K.forward_kinematics(model, q)
    fids = list(frame_ids)
    T = K.frame_placements(model, oMi, fids)
    xi = lie.se3_log(lie.se3_compose(lie.se3_inverse(targets), T))               # (B, nf, 6)
    w = np.broadcast_to(np.asarray(weights, dtype=np.float64), xi.shape[:-1])
    Jr = lie.right_jacobian_se3(xi, terms=40)
    g = 2.0 * w[..., None] * np.einsum("...ji,...j->...i", np.linalg.inv(Jr), xi)  # Jr^-T xi
    R = lie.quat_to_matrix(T[..., 3:7])
    f_lin = np.einsum("...ij,...j->...i", R, g[..., :3])
    f_ang = np.cross(T[..., :3], f_lin) + np.einsum("...ij,...j->...i", R, g[..., 3:])
    F = np.concatenate([f_lin, f_ang], -1)                                       # (B, nf, 6)
    gv = np.zeros((B, model.nv))
    for j in range(model.njoints):
        nvj = int(model.nvs[j])
        if nvj == 0:
            continue
        S = K._joint_world_columns(model, oMi, q, j)                            # (B, 6, nvj)
        moved = [i for i, f in enumerate(fids) if j in model.supports[model.frames[f].parent_joint]]
        if moved:
            iv = int(model.idx_vs[j])
            gv[:, iv:iv + nvj] = np.einsum("bkc,bfk->bc", S, F[:, moved])
    gq = np.zeros_like(q)
    for j, jm in enumerate(model.joint_models):
        nvj = int(model.nvs[j])
        if nvj == 0:
            continue
        iq, iv = int(model.idx_qs[j]), int(model.idx_vs[j])
        kind = jm.kind
        if kind.startswith("revolute") and kind != "revolute_unbounded" or kind.startswith("prismatic") \
                or kind == "translation":
            gq[:, iq:iq + nvj] = gv[:, iv:iv + nvj]
        elif kind == "revolute_unbounded":
            c, s = q[:, iq], q[:, iq + 1]
            r2 = np.maximum(c * c + s * s, 1e-300)
            gq[:, iq] = -gv[:, iv] * s / r2
            gq[:, iq + 1] = gv[:, iv] * c / r2
        elif kind == "planar":
            c, s = q[:, iq + 2], q[:, iq + 3]
            hc = np.sqrt(np.maximum((1.0 + c) / 2.0, 0.0))
            hs = np.sqrt(np.maximum((1.0 - c) / 2.0, 0.0)) * np.sign(s)
            ct, st = hc * hc - hs * hs, 2.0 * hs * hc
            g0, g1, g2 = gv[:, iv], gv[:, iv + 1], gv[:, iv + 2]
            gq[:, iq] = ct * g0 - st * g1
            gq[:, iq + 1] = st * g0 + ct * g1
            gq[:, iq + 2] = -g2 / st
            gq[:, iq + 3] = 0.0
        elif kind in ("free_flyer", "spherical"):
            ff = kind == "free_flyer"
            qo, vo = (iq + 3, iv + 3) if ff else (iq, iv)
            qr = q[:, qo:qo + 4]
            n = np.linalg.norm(qr, axis=-1, keepdims=True)
            u = qr / n
            ga = gv[:, vo:vo + 3]
            # delta_ang = M du with M = 2 [u_w I - hat(u_v) | -u_v]; dL/du = M^T ga
            h = 2.0 * np.concatenate([u[:, 3:4] * ga + np.cross(u[:, :3], ga),
                                      -np.sum(u[:, :3] * ga, -1, keepdims=True)], -1)
            gq[:, qo:qo + 4] = (h - u * np.sum(u * h, -1, keepdims=True)) / n
            if ff:
                Rj = lie.quat_to_matrix(u)
                gq[:, iq:iq + 3] = np.einsum("bij,bj->bi", Rj, gv[:, iv:iv + 3])
        else:
            raise NotImplementedError(kind)
    return gq

"""IK residual stack and Levenberg-Marquardt / Gauss-Newton in float64 — oracle only.

Restates, vectorised over independent problems that share one robot and one
target-frame list:

* the stack ``solve_ik`` builds (``src/better_robot/tasks/ik.py:191-209``):
  one ``PoseResidual`` per target (``residuals/pose.py:58-103``), then
  ``JointPositionLimit`` with item weight ``limit_weight`` (``residuals/limits.py:56-86``),
  then ``RestResidual`` with item weight ``rest_weight`` (``residuals/regularization.py:48-64``);
* ``LevenbergMarquardt.minimize`` (``optim/optimizers/levenberg_marquardt.py:61-135``)
  with ``Adaptive`` damping (``optim/strategies/adaptive.py:9-25``) and the
  ``Cholesky`` solver with least-squares fallback (``optim/solvers/cholesky.py:14-20``);
* ``GaussNewton.minimize`` (``optim/optimizers/gauss_newton.py:27-76``).

The float64 run bypasses ``solve_ik``'s ``.float()`` cast (``tasks/ik.py:186``) by
building the same problem directly, as the reference itself does internally.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import kinematics as K
from . import lie


@dataclass
class IKSettings:
    pos_weight: float = 1.0
    ori_weight: float = 1.0
    limit_weight: float = 0.1
    rest_weight: float = 0.01
    lam0: float = 1e-3
    factor: float = 10.0
    tol: float = 1e-6
    max_iter: int = 50
    optimizer: str = "lm"          # "lm" | "gn"
    gn_eps: float = 1e-8
    lam_min: float = 1e-10         # Adaptive.accept floor, adaptive.py:19
    lam_max: float = 1e8           # Adaptive.reject cap, adaptive.py:23
    kernel: str = "l2"             # "l2" | "huber" | "cauchy" | "tukey" (tasks/ik.py:116-133)
    kernel_param: float | None = None  # delta (huber) or c (cauchy, tukey); None = the class default


KERNEL_DEFAULTS = {"huber": 1.0, "cauchy": 1.0, "tukey": 4.685}  # optim/kernels/{huber,cauchy,tukey}.py


def kernel_weight(name: str, s: np.ndarray, param: float | None = None) -> np.ndarray:
    """IRLS weight w(s) of a squared residual row ``s`` (``optim/kernels/*.py: weight``)."""
    if name == "l2":
        return np.ones_like(s)
    c = KERNEL_DEFAULTS[name] if param is None else param
    if name == "huber":                        # huber.py: min(1, delta / sqrt(s))
        s = np.maximum(s, 0.0)
        return np.where(s <= c * c, 1.0, c / np.sqrt(s + 1e-30))
    if name == "cauchy":                       # cauchy.py: 1 / (1 + s / c^2)
        return 1.0 / (1.0 + s / (c * c))
    if name == "tukey":                        # tukey.py: max(1 - s / c^2, 0)^2
        u = np.maximum(1.0 - s / (c * c), 0.0)
        return u * u
    raise ValueError(f"unknown kernel {name!r}")


def _np(x):
    return K._np(x)


def residual_and_jacobian(model, q, frame_ids, targets, q_rest, s: IKSettings, want_jac: bool = True, kinds=None):
    """Stacked residual ``(P, dim)`` and Jacobian ``(P, dim, nv)`` of the IK cost stack at ``q (P, nq)``.

    ``targets (P, k, 7)`` are the per-problem target poses of ``frame_ids`` (length k);
    ``kinds[i]`` is "pose" (default, ``PoseResidual`` with pos / ori weights), "position"
    (``PositionResidual``, weight ``pos_weight``) or "orientation" (``OrientationResidual``,
    weight ``ori_weight``), ``residuals/pose.py:58-195``.
    """
    q = _np(q)
    oMi, _ = K.forward_kinematics(model, q)
    w = np.array([s.pos_weight] * 3 + [s.ori_weight] * 3)
    rs, Js = [], []
    for i, f in enumerate(frame_ids):
        Tt = targets[:, i, :]
        fr = model.frames[f]
        Tee = lie.se3_compose(oMi[:, fr.parent_joint, :], _np(fr.joint_placement))
        kind = "pose" if kinds is None else kinds[i]
        if kind == "position":                                            # pose.py:127-141
            rs.append((Tee[:, :3] - Tt[:, :3]) * s.pos_weight)
            if want_jac:
                Jlwa = K.frame_jacobian(model, oMi, q, f, "local_world_aligned")
                Js.append(Jlwa[:, :3] * s.pos_weight)
            continue
        if kind == "orientation":                                         # pose.py:165-195
            r = lie.so3_log(lie.quat_mul(lie.so3_inverse(Tt[:, 3:7]), Tee[:, 3:7]))
            rs.append(r * s.ori_weight)
            if want_jac:
                Jlwa = K.frame_jacobian(model, oMi, q, f, "local_world_aligned")
                RT = np.swapaxes(lie.quat_to_matrix(Tee[:, 3:7]), -1, -2)
                Js.append(lie.right_jacobian_inv_so3(r) @ (RT @ Jlwa[:, 3:]) * s.ori_weight)
            continue
        xi = lie.se3_log(lie.se3_compose(lie.se3_inverse(Tt), Tee))       # pose.py:63-64
        rs.append(xi * w)
        if want_jac:
            Jlwa = K.frame_jacobian(model, oMi, q, f, "local_world_aligned")  # pose.py:85
            RT = np.swapaxes(lie.quat_to_matrix(Tee[:, 3:7]), -1, -2)
            Jloc = np.concatenate([RT @ Jlwa[:, :3], RT @ Jlwa[:, 3:]], -2)  # pose.py:91-95
            Js.append((lie.right_jacobian_inv_se3(xi) @ Jloc) * w[:, None])  # pose.py:98-103
    lo = _np(model.lower_pos_limit)
    hi = _np(model.upper_pos_limit)
    if s.limit_weight > 0.0:
        with np.errstate(invalid="ignore"):
            rl = np.concatenate([np.maximum(lo - q, 0.0), np.maximum(q - hi, 0.0)], -1)
        rs.append(np.nan_to_num(rl, nan=0.0, posinf=0.0, neginf=0.0) * s.limit_weight)
        if want_jac:
            dq_dv = np.zeros((model.nq, model.nv))                        # limits.py:40-49
            for j, jm in enumerate(model.joint_models):
                if jm.nq == 0 or jm.nq != jm.nv:
                    continue
                for k in range(jm.nq):
                    dq_dv[model.idx_qs[j] + k, model.idx_vs[j] + k] = 1.0
            ld = np.where(q < lo, -1.0, 0.0)
            ud = np.where(q > hi, 1.0, 0.0)
            Jl = np.concatenate([ld[..., None] * dq_dv, ud[..., None] * dq_dv], -2)
            Js.append(Jl * s.limit_weight)
    if s.rest_weight > 0.0:
        rs.append(K.difference(model, np.broadcast_to(_np(q_rest), q.shape), q) * s.rest_weight)
        if want_jac:
            Js.append(np.broadcast_to(np.eye(model.nv), q.shape[:-1] + (model.nv, model.nv)) * s.rest_weight)
    r = np.concatenate(rs, -1)
    J = np.concatenate(Js, -2) if want_jac else None
    return r, J


def _solve(H: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Cholesky solve with least-squares fallback per problem (``cholesky.py:14-20``)."""
    out = np.empty_like(b)
    try:
        L = np.linalg.cholesky(H)
        y = np.linalg.solve(L, b[..., None])
        return np.linalg.solve(np.swapaxes(L, -1, -2), y)[..., 0]
    except np.linalg.LinAlgError:
        for p in range(H.shape[0]):
            try:
                L = np.linalg.cholesky(H[p])
                out[p] = np.linalg.solve(L.T, np.linalg.solve(L, b[p]))
            except np.linalg.LinAlgError:
                out[p] = np.linalg.lstsq(H[p], b[p], rcond=None)[0]
        return out


@dataclass
class IKOutcome:
    q: np.ndarray          # (P, nq)
    residual: np.ndarray   # (P, dim)
    cost: np.ndarray       # (P,)   0.5 |r|^2
    iters: np.ndarray      # (P,)   int
    converged: np.ndarray  # (P,)   bool
    # (P,) smallest |cost_new - cost| in units of the cost's float64 spacing over the accept
    # tests that decide convergence (pre-step |J^T r| < tol); inf if there was none.  A few
    # units mean the verdict was decided by the rounding of a float64 sum: any implementation
    # that sums in another order (BetterRobot's torch code included) flips it at random.
    margin: np.ndarray | None = None


def solve(model, frame_ids, targets, q0, s: IKSettings, q_rest=None, kinds=None) -> IKOutcome:
    """Run LM (or GN) on ``P`` independent problems; each follows the single-instance reference loop."""
    q = _np(q0).copy()
    P = q.shape[0]
    targets = _np(targets)
    q_rest = _np(model.q_neutral) if q_rest is None else _np(q_rest)
    lo = _np(model.lower_pos_limit)
    hi = _np(model.upper_pos_limit)
    r, _ = residual_and_jacobian(model, q, frame_ids, targets, q_rest, s, want_jac=False, kinds=kinds)
    cost = 0.5 * np.sum(r * r, -1)
    lam = np.full(P, s.lam0 if s.optimizer == "lm" else 0.0)
    active = np.ones(P, dtype=bool)
    iters = np.full(P, s.max_iter, dtype=np.int64)
    conv = np.zeros(P, dtype=bool)
    margin = np.full(P, np.inf)
    nv = model.nv
    for it in range(s.max_iter):
        idx = np.nonzero(active)[0]
        if idx.size == 0:
            break
        qa = q[idx]
        _, J = residual_and_jacobian(model, qa, frame_ids, targets[idx], q_rest, s, kinds=kinds)
        ra = r[idx]
        if s.kernel != "l2":  # IRLS: rows scaled by sqrt(w(r_i^2)) (levenberg_marquardt.py:27-44)
            sw = np.sqrt(np.maximum(kernel_weight(s.kernel, ra * ra, s.kernel_param), 0.0))
            ra = ra * sw
            J = J * sw[..., None]
        JtJ = np.swapaxes(J, -1, -2) @ J
        Jtr = (np.swapaxes(J, -1, -2) @ ra[..., None])[..., 0]
        damp = lam[idx] if s.optimizer == "lm" else np.full(idx.size, s.gn_eps)
        H = JtJ + damp[:, None, None] * np.eye(nv)
        dv = _solve(H, -Jtr)
        qn = K.integrate(model, qa, dv)
        qn = np.minimum(np.maximum(qn, lo), hi)
        rn, _ = residual_and_jacobian(model, qn, frame_ids, targets[idx], q_rest, s, want_jac=False, kinds=kinds)
        cn = 0.5 * np.sum(rn * rn, -1)
        gnorm = np.linalg.norm(Jtr, axis=-1)
        ulps = np.abs(cn - cost[idx]) / np.spacing(np.maximum(cn, cost[idx]))
        dec = gnorm < s.tol
        margin[idx[dec]] = np.minimum(margin[idx[dec]], ulps[dec])
        if s.optimizer == "lm":
            acc = cn < cost[idx]
            a_idx = idx[acc]
            q[a_idx] = qn[acc]
            r[a_idx] = rn[acc]
            cost[a_idx] = cn[acc]
            lam[a_idx] = np.maximum(lam[a_idx] / s.factor, s.lam_min)
            rej = idx[~acc]
            lam[rej] = np.minimum(lam[rej] * s.factor, s.lam_max)
            done = acc & (gnorm < s.tol)
        else:
            q[idx] = qn
            r[idx] = rn
            cost[idx] = cn
            done = gnorm < s.tol
        d_idx = idx[done]
        conv[d_idx] = True
        iters[d_idx] = it + 1
        active[d_idx] = False
    return IKOutcome(q=q, residual=r, cost=cost, iters=iters, converged=conv, margin=margin)


def pose_errors(model, q, frame_ids, targets):
    """Per-problem max position error (m) and rotation error (rad) over the targets."""
    oMi, _ = K.forward_kinematics(model, _np(q))
    targets = _np(targets)
    pe = np.zeros(oMi.shape[0])
    re = np.zeros(oMi.shape[0])
    for i, f in enumerate(frame_ids):
        fr = model.frames[f]
        Tee = lie.se3_compose(oMi[:, fr.parent_joint, :], _np(fr.joint_placement))
        Terr = lie.se3_compose(lie.se3_inverse(targets[:, i]), Tee)
        pe = np.maximum(pe, np.linalg.norm(Tee[:, :3] - targets[:, i, :3], axis=-1))
        re = np.maximum(re, np.linalg.norm(lie.so3_log(Terr[:, 3:7]), axis=-1))
    return pe, re

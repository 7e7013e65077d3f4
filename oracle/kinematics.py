"""Forward kinematics and Jacobians in float64 numpy — oracle only.

Restates ``src/better_robot/kinematics/forward.py`` and
``src/better_robot/kinematics/jacobian.py`` for the joint kinds of
``src/better_robot/data_model/joint_models/``: universe/fixed, revolute about any axis,
revolute_unbounded, prismatic, free-flyer, spherical, planar, translation.
"""

from __future__ import annotations

import numpy as np

from . import lie

_AXES = {"revolute_rx": (1, 0, 0), "revolute_ry": (0, 1, 0), "revolute_rz": (0, 0, 1),
         "prismatic_px": (1, 0, 0), "prismatic_py": (0, 1, 0), "prismatic_pz": (0, 0, 1)}


def _np(x) -> np.ndarray:
    if hasattr(x, "detach"):
        return x.detach().cpu().double().numpy()
    return np.asarray(x, dtype=np.float64)


def axis_of(jm) -> np.ndarray:
    if jm.kind in _AXES:
        return np.array(_AXES[jm.kind], dtype=np.float64)
    return _np(jm.axis).reshape(3)


def joint_transform(jm, qj: np.ndarray) -> np.ndarray:
    """``JointModel.joint_transform`` for the supported kinds.

    revolute: ``se3_from_axis_angle`` (``revolute.py:18-21``, ``_torch_native_backend.py:345-348``);
    prismatic: pure translation ``d * axis``; free-flyer: ``se3_normalize(q)`` (``free_flyer.py:31-36``).
    """
    kind = jm.kind
    batch = qj.shape[:-1]
    if kind == "revolute_unbounded":                  # revolute.py:206-211: angle = atan2(sin, cos)
        a = axis_of(jm)
        half = np.arctan2(qj[..., 1], qj[..., 0]) / 2.0
        q = np.concatenate([np.sin(half)[..., None] * a, np.cos(half)[..., None]], -1)
        return np.concatenate([np.zeros(batch + (3,)), q], -1)
    if kind == "spherical":                           # spherical.py:22-32: rotation normalize(q)
        return np.concatenate([np.zeros(batch + (3,)), lie.so3_normalize(qj)], -1)
    if kind == "planar":                              # planar.py:20-41: half-angle from cos, sign of sin
        c, s = qj[..., 2], qj[..., 3]
        hc = np.sqrt(np.maximum((1.0 + c) / 2.0, 0.0))
        hs = np.sqrt(np.maximum((1.0 - c) / 2.0, 0.0)) * np.sign(s)
        z = np.zeros_like(c)
        return np.stack([qj[..., 0], qj[..., 1], z, z, z, hs, hc], -1)
    if kind == "translation":                         # translation.py:19-23
        return np.concatenate([qj[..., :3], np.zeros(batch + (3,)), np.ones(batch + (1,))], -1)
    if kind.startswith("revolute"):
        a = axis_of(jm)
        half = qj[..., 0] / 2.0
        q = np.concatenate([np.sin(half)[..., None] * a, np.cos(half)[..., None]], -1)
        return np.concatenate([np.zeros(batch + (3,)), q], -1)
    if kind.startswith("prismatic"):
        a = axis_of(jm)
        t = qj[..., 0:1] * a
        return np.concatenate([t, np.zeros(batch + (3,)), np.ones(batch + (1,))], -1)
    if kind == "free_flyer":
        return lie.se3_normalize(qj)
    raise NotImplementedError(kind)


def forward_kinematics(model, q) -> tuple[np.ndarray, np.ndarray]:
    """``forward_kinematics_raw`` (``forward.py:73-135``): returns ``(oMi, liMi)`` ``(B..., nj, 7)``."""
    q = _np(q)
    batch = q.shape[:-1]
    P = _np(model.joint_placements)
    nj = model.njoints
    world = [None] * nj
    local = [None] * nj
    ident = np.broadcast_to(np.array([0, 0, 0, 0, 0, 0, 1.0]), batch + (7,))
    for j in model.topo_order:
        nq = model.nqs[j]
        if nq > 0:
            Tj = joint_transform(model.joint_models[j], q[..., model.idx_qs[j]:model.idx_qs[j] + nq])
        else:
            Tj = ident
        loc = lie.se3_compose(np.broadcast_to(P[j], batch + (7,)), Tj)
        local[j] = loc
        p = model.parents[j]
        world[j] = loc if p < 0 else lie.se3_compose(world[p], loc)
    return np.stack(world, -2), np.stack(local, -2)


def frame_placements(model, oMi: np.ndarray, frame_ids=None) -> np.ndarray:
    """``update_frame_placements`` (``forward.py:194-219``) for ``frame_ids`` (default: all)."""
    ids = range(model.nframes) if frame_ids is None else frame_ids
    out = []
    for f in ids:
        fr = model.frames[f]
        out.append(lie.se3_compose(oMi[..., fr.parent_joint, :], _np(fr.joint_placement)))
    return np.stack(out, -2)


def _joint_world_columns(model, oMi: np.ndarray, q: np.ndarray, j: int) -> np.ndarray:
    """``Ad(oMi_j) S_j``: ``[R S_lin + hat(p) R S_ang; R S_ang]`` (``jacobian.py:30-79``). ``(B..., 6, nv_j)``."""
    jm = model.joint_models[j]
    T = oMi[..., j, :]
    p = T[..., :3]
    R = lie.quat_to_matrix(T[..., 3:7])
    if jm.kind.startswith("revolute"):               # incl. revolute_unbounded (revolute.py:213-216)
        S = np.zeros((6, 1)); S[3:, 0] = axis_of(jm)
    elif jm.kind == "spherical":                     # spherical.py:34-41
        S = np.zeros((6, 3)); S[3:, :] = np.eye(3)
    elif jm.kind == "planar":                        # planar.py:43-50
        S = np.zeros((6, 3)); S[0, 0] = 1.0; S[1, 1] = 1.0; S[5, 2] = 1.0
    elif jm.kind == "translation":                   # translation.py:25-32
        S = np.zeros((6, 3)); S[:3, :] = np.eye(3)
    elif jm.kind.startswith("prismatic"):
        S = np.zeros((6, 1)); S[:3, 0] = axis_of(jm)
    elif jm.kind == "free_flyer":
        S = np.eye(6)
    else:
        raise NotImplementedError(jm.kind)
    RSl = R @ S[:3]
    RSa = R @ S[3:]
    return np.concatenate([RSl + lie.hat(p) @ RSa, RSa], -2)


def compute_joint_jacobians(model, oMi: np.ndarray, q) -> np.ndarray:
    """World joint Jacobians ``(B..., nj, 6, nv)`` by parent-copy propagation (``jacobian.py:30-79``)."""
    q = _np(q)
    batch = q.shape[:-1]
    J = np.zeros(batch + (model.njoints, 6, model.nv))
    for j in model.topo_order:
        p = model.parents[j]
        if p >= 0:
            J[..., j, :, :] = J[..., p, :, :]
        nv = model.nvs[j]
        if nv == 0:
            continue
        v = model.idx_vs[j]
        J[..., j, :, v:v + nv] = _joint_world_columns(model, oMi, q, j)
    return J


def frame_jacobian(model, oMi: np.ndarray, q, frame_id: int, reference: str = "local_world_aligned") -> np.ndarray:
    """``get_frame_jacobian`` (``jacobian.py:129-227``) via the support loop. ``(B..., 6, nv)``."""
    q = _np(q)
    batch = q.shape[:-1]
    fr = model.frames[frame_id]
    Jp = np.zeros(batch + (6, model.nv))
    for j in model.supports[fr.parent_joint]:
        nv = model.nvs[j]
        if nv == 0:
            continue
        v = model.idx_vs[j]
        Jp[..., :, v:v + nv] = _joint_world_columns(model, oMi, q, j)
    if reference == "world":
        return Jp
    Tf = lie.se3_compose(oMi[..., fr.parent_joint, :], _np(fr.joint_placement))
    lin = Jp[..., :3, :] - lie.hat(Tf[..., :3]) @ Jp[..., 3:, :]
    Jlwa = np.concatenate([lin, Jp[..., 3:, :]], -2)
    if reference == "local_world_aligned":
        return Jlwa
    if reference == "local":
        RT = np.swapaxes(lie.quat_to_matrix(Tf[..., 3:7]), -1, -2)
        return np.concatenate([RT @ Jlwa[..., :3, :], RT @ Jlwa[..., 3:, :]], -2)
    raise ValueError(reference)


def integrate(model, q, v) -> np.ndarray:
    """``Model.integrate`` (``model.py:160-174``): revolute/prismatic ``q+v``, free-flyer ``normalize(q . exp(v))``."""
    q = _np(q)
    v = _np(v)
    parts = []
    for j, jm in enumerate(model.joint_models):
        if jm.nq == 0:
            continue
        iq, iv = model.idx_qs[j], model.idx_vs[j]
        qj = q[..., iq:iq + jm.nq]
        vj = v[..., iv:iv + jm.nv]
        if jm.kind == "free_flyer":
            parts.append(lie.se3_normalize(lie.se3_compose(qj, lie.se3_exp(vj))))
        elif jm.kind == "spherical":                 # spherical.py:52-56
            parts.append(lie.so3_normalize(lie.quat_mul(qj, lie.so3_exp(vj))))
        elif jm.kind == "revolute_unbounded":        # revolute.py:223-231
            th = np.arctan2(qj[..., 1], qj[..., 0]) + vj[..., 0]
            parts.append(np.stack([np.cos(th), np.sin(th)], -1))
        elif jm.kind == "planar":                    # planar.py:61-68
            th = np.arctan2(qj[..., 3], qj[..., 2]) + vj[..., 2]
            parts.append(np.stack([qj[..., 0] + vj[..., 0], qj[..., 1] + vj[..., 1], np.cos(th), np.sin(th)], -1))
        else:
            parts.append(qj + vj)
    return np.concatenate(parts, -1) if parts else q.copy()


def difference(model, q0, q1) -> np.ndarray:
    """``Model.difference`` (``model.py:176-190``): ``q1 - q0``; free-flyer ``log(q0^-1 q1)``."""
    q0 = _np(q0)
    q1 = _np(q1)
    parts = []
    for j, jm in enumerate(model.joint_models):
        if jm.nq == 0:
            continue
        iq = model.idx_qs[j]
        a = q0[..., iq:iq + jm.nq]
        b = q1[..., iq:iq + jm.nq]
        if jm.kind == "free_flyer":
            parts.append(lie.se3_log(lie.se3_compose(lie.se3_inverse(a), b)))
        elif jm.kind == "spherical":                 # spherical.py:58-62
            parts.append(lie.so3_log(lie.so3_normalize(lie.quat_mul(lie.so3_inverse(a), b))))
        elif jm.kind == "revolute_unbounded":        # revolute.py:233-237
            parts.append((np.arctan2(b[..., 1], b[..., 0]) - np.arctan2(a[..., 1], a[..., 0]))[..., None])
        elif jm.kind == "planar":                    # planar.py:70-76
            parts.append(np.stack([b[..., 0] - a[..., 0], b[..., 1] - a[..., 1],
                                   np.arctan2(b[..., 3], b[..., 2]) - np.arctan2(a[..., 3], a[..., 2])], -1))
        else:
            parts.append(b - a)
    return np.concatenate(parts, -1)

"""Seeded synthetic robots and workloads for the five benchmark configurations.

No URDF or dataset is involved: every robot is built from a seeded description
(joint tree, parent-to-joint offsets, limits, tracked frames), exactly as one
would with the reference's ``ModelBuilder`` (``src/better_robot/io/parsers/programmatic.py:67-423``).
The same description can be handed to that builder to produce the reference
``Model`` with identical joint and frame numbering.

* ``chain7``   — serial 7-revolute chain, axes local z, offsets t~U[-0.15,0.15]^3,
  rotations uniform on S^3, limits +-2.8 rad, one end-effector frame ``ee``.
* ``humanoid`` — free-flyer base + 30 revolute joints in five branches of
  6, 6, 7, 7, 4 (legs, arms, torso/head), 12 tracked frames.
* ``dual_arm`` — fixed base with two 7-revolute chains (14 DOF), frames ``ee_l``/``ee_r``.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from .model import Model, build_model

LIMIT = 2.8


def _rand_pose(rng: np.random.Generator) -> list[float]:
    t = rng.uniform(-0.15, 0.15, size=3)
    q = rng.normal(size=4)
    q = q / np.linalg.norm(q)
    return [*t.tolist(), *q.tolist()]


def chain_spec(seed: int = 0, n: int = 7, name: str = "chain7") -> dict:
    """Serial chain: fixed root, ``n`` revolute-z joints, one tool frame ``ee``."""
    rng = np.random.default_rng(seed)
    joints = [{"name": "root_joint", "kind": "fixed", "parent": 0, "body": "base"}]
    for i in range(n):
        joints.append({"name": f"j{i + 1}", "kind": "revolute_rz", "parent": i + 1,
                       "origin": _rand_pose(rng), "lower": -LIMIT, "upper": LIMIT,
                       "body": f"link{i + 1}"})
    frames = [{"name": "ee", "parent": n + 1, "placement": _rand_pose(rng)}]
    return {"name": name, "joints": joints, "frames": frames}


def floating_chain_spec(seed: int = 4, n: int = 4) -> dict:
    """Floating-base chain: free-flyer root, ``n`` revolute-z joints, one tool frame ``ee``
    (a floating-base robot small enough for the reference's dense trajectory solver)."""
    rng = np.random.default_rng(seed)
    joints = [{"name": "root_joint", "kind": "free_flyer", "parent": 0, "body": "base"}]
    for i in range(n):
        joints.append({"name": f"j{i + 1}", "kind": "revolute_rz", "parent": i + 1,
                       "origin": _rand_pose(rng), "lower": -LIMIT, "upper": LIMIT,
                       "body": f"link{i + 1}"})
    frames = [{"name": "ee", "parent": n + 1, "placement": _rand_pose(rng)}]
    return {"name": "floating_chain", "joints": joints, "frames": frames}


def dual_arm_spec(seed: int = 2, n: int = 7) -> dict:
    """Fixed base with two ``n``-revolute chains; tool frames ``ee_l`` and ``ee_r``."""
    rng = np.random.default_rng(seed)
    joints = [{"name": "root_joint", "kind": "fixed", "parent": 0, "body": "torso"}]
    tips = []
    for side in ("l", "r"):
        parent = 1
        for i in range(n):
            joints.append({"name": f"{side}{i + 1}", "kind": "revolute_rz", "parent": parent,
                           "origin": _rand_pose(rng), "lower": -LIMIT, "upper": LIMIT,
                           "body": f"{side}_link{i + 1}"})
            parent = len(joints)
        tips.append(parent)
    frames = [{"name": "ee_l", "parent": tips[0], "placement": _rand_pose(rng)},
              {"name": "ee_r", "parent": tips[1], "placement": _rand_pose(rng)}]
    return {"name": "dual_arm", "joints": joints, "frames": frames}


def mixed_spec(seed: int = 3) -> dict:
    """A mobile manipulator using every multi-slot joint kind: fixed root, planar base,
    3-DOF translation lift, revolute-z, spherical shoulder, revolute-y, unbounded wrist
    (axis x); frames ``ee`` (wrist) and ``mid`` (shoulder)."""
    rng = np.random.default_rng(seed)
    kinds = [("planar", "mobile"), ("translation", "lift"), ("revolute_rz", "link1"), ("spherical", "link2"),
             ("revolute_ry", "link3"), ("revolute_unbounded", "link4")]
    joints = [{"name": "root_joint", "kind": "fixed", "parent": 0, "body": "base"}]
    for i, (kind, body) in enumerate(kinds):
        rec = {"name": f"j_{body}", "kind": kind, "parent": i + 1, "origin": _rand_pose(rng), "body": body}
        if kind.startswith("revolute_r"):
            rec.update(lower=-LIMIT, upper=LIMIT)
        if kind == "revolute_unbounded":
            rec["axis"] = (1.0, 0.0, 0.0)
        joints.append(rec)
    frames = [{"name": "ee", "parent": len(joints), "placement": _rand_pose(rng)},
              {"name": "mid", "parent": 5, "placement": _rand_pose(rng)}]
    return {"name": "mixed", "joints": joints, "frames": frames}


HUMANOID_BRANCHES = (("lleg", 6), ("rleg", 6), ("larm", 7), ("rarm", 7), ("torso", 4))


def humanoid_spec(seed: int = 1, n_tracked: int = 12) -> dict:
    """Free-flyer pelvis + 30 revolute joints in 5 branches; ``n_tracked`` op frames.

    Tracked frames: the leaf link of each branch (5), then ``n_tracked - 5``
    mid-branch links drawn without replacement by the seed; each frame has a
    random offset placement.
    """
    rng = np.random.default_rng(seed)
    joints = [{"name": "root_joint", "kind": "free_flyer", "parent": 0, "body": "pelvis"}]
    leaves, mids = [], []
    for bname, length in HUMANOID_BRANCHES:
        parent = 1
        for i in range(length):
            joints.append({"name": f"{bname}{i + 1}", "kind": "revolute_rz", "parent": parent,
                           "origin": _rand_pose(rng), "lower": -LIMIT, "upper": LIMIT,
                           "body": f"{bname}_link{i + 1}"})
            parent = len(joints)
            (leaves if i == length - 1 else mids).append(parent)
    n_mid = max(0, n_tracked - len(leaves))
    pick = sorted(rng.choice(len(mids), size=n_mid, replace=False).tolist())
    tracked = leaves + [mids[i] for i in pick]
    frames = [{"name": f"track{k}", "parent": jid, "placement": _rand_pose(rng)}
              for k, jid in enumerate(tracked[:n_tracked])]
    return {"name": "humanoid", "joints": joints, "frames": frames}


def model_from_spec(spec: dict, dtype: torch.dtype = torch.float32) -> Model:
    return build_model(spec["name"], spec["joints"], spec["frames"], dtype=dtype)


def op_frame_ids(model: Model) -> list[int]:
    """Ids of the operational (non-body) frames, in declaration order."""
    return [i for i, f in enumerate(model.frames) if f.frame_type != "body"]


def random_q(model: Model, batch: int, seed: int, rev_range: float = LIMIT,
             base_translation: float = 0.0) -> torch.Tensor:
    """Configurations ``(batch, nq)`` in float64: revolute uniform in +-``rev_range``,
    free-flyer translation uniform in +-``base_translation``, quaternion uniform on S^3."""
    rng = np.random.default_rng(seed)
    q = np.zeros((batch, model.nq))
    for j, jm in enumerate(model.joint_models):
        iq = model.idx_qs[j]
        if jm.kind == "free_flyer":
            q[:, iq:iq + 3] = rng.uniform(-base_translation, base_translation, size=(batch, 3))
            quat = rng.normal(size=(batch, 4))
            q[:, iq + 3:iq + 7] = quat / np.linalg.norm(quat, axis=1, keepdims=True)
        elif jm.kind == "spherical":
            quat = rng.normal(size=(batch, 4))
            q[:, iq:iq + 4] = quat / np.linalg.norm(quat, axis=1, keepdims=True)
        elif jm.kind == "planar":
            th = rng.uniform(-np.pi, np.pi, size=batch)
            q[:, iq:iq + 2] = rng.uniform(-0.5, 0.5, size=(batch, 2))
            q[:, iq + 2], q[:, iq + 3] = np.cos(th), np.sin(th)
        elif jm.kind == "revolute_unbounded":
            th = rng.uniform(-np.pi, np.pi, size=batch)
            q[:, iq], q[:, iq + 1] = np.cos(th), np.sin(th)
        elif jm.kind == "translation":
            q[:, iq:iq + 3] = rng.uniform(-0.3, 0.3, size=(batch, 3))
        elif jm.nq == 1:
            q[:, iq] = rng.uniform(-rev_range, rev_range, size=batch)
    return torch.from_numpy(q)


def random_targets(batch: int, nframes: int, seed: int, t_range: float = 0.5) -> torch.Tensor:
    """Random SE3 poses ``(batch, nframes, 7)`` float64: t~U(+-t_range), quaternion uniform."""
    rng = np.random.default_rng(seed)
    t = rng.uniform(-t_range, t_range, size=(batch, nframes, 3))
    quat = rng.normal(size=(batch, nframes, 4))
    quat /= np.linalg.norm(quat, axis=-1, keepdims=True)
    return torch.from_numpy(np.concatenate([t, quat], axis=-1))


def noisy_start(model: Model, q_star: torch.Tensor, sigma: float, seed: int) -> torch.Tensor:
    """``q* (+) noise``, clamped to the joint limits (float64).

    Revolute joints get N(0, sigma^2) rad.  A free-flyer base gets a rotation
    ``exp(w)`` with w ~ N(0, sigma^2) per axis composed on the right of its
    quaternion, and N(0, (sigma/3)^2) m added to its translation.
    """
    rng = np.random.default_rng(seed)
    q = q_star.detach().cpu().double().numpy().copy()
    lo = model.lower_pos_limit.double().numpy()
    hi = model.upper_pos_limit.double().numpy()
    for j, jm in enumerate(model.joint_models):
        iq = model.idx_qs[j]
        if jm.kind == "free_flyer":
            q[:, iq:iq + 3] += rng.normal(0.0, sigma / 3.0, size=(q.shape[0], 3))
            w = rng.normal(0.0, sigma, size=(q.shape[0], 3))
            th = np.linalg.norm(w, axis=1, keepdims=True)
            s = np.where(th > 1e-12, np.sin(0.5 * th) / np.maximum(th, 1e-12), 0.5)
            dq = np.concatenate([s * w, np.cos(0.5 * th)], axis=1)
            q[:, iq + 3:iq + 7] = _quat_mul_np(q[:, iq + 3:iq + 7], dq)
        elif jm.kind == "spherical":
            w = rng.normal(0.0, sigma, size=(q.shape[0], 3))
            th = np.linalg.norm(w, axis=1, keepdims=True)
            s = np.where(th > 1e-12, np.sin(0.5 * th) / np.maximum(th, 1e-12), 0.5)
            q[:, iq:iq + 4] = _quat_mul_np(q[:, iq:iq + 4], np.concatenate([s * w, np.cos(0.5 * th)], axis=1))
        elif jm.kind in ("planar", "revolute_unbounded"):
            k = iq + (2 if jm.kind == "planar" else 0)
            th = np.arctan2(q[:, k + 1], q[:, k]) + rng.normal(0.0, sigma, size=q.shape[0])
            q[:, k], q[:, k + 1] = np.cos(th), np.sin(th)
            if jm.kind == "planar":
                q[:, iq:iq + 2] += rng.normal(0.0, sigma / 3.0, size=(q.shape[0], 2))
        elif jm.kind == "translation":
            q[:, iq:iq + 3] += rng.normal(0.0, sigma / 3.0, size=(q.shape[0], 3))
        elif jm.nq == 1:
            q[:, iq] = np.clip(q[:, iq] + rng.normal(0.0, sigma, size=q.shape[0]), lo[iq], hi[iq])
    return torch.from_numpy(q)


def _quat_mul_np(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ax, ay, az, aw = a[:, 0], a[:, 1], a[:, 2], a[:, 3]
    bx, by, bz, bw = b[:, 0], b[:, 1], b[:, 2], b[:, 3]
    return np.stack([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz], axis=1)


def trajopt_endpoints(model: Model, n: int, seed: int, spread: float = 1.0):
    """Start and goal configurations (float64) for trajectory problems: start uniform in
    +-2.5 rad, goal = start + U(+-spread) per joint, both clamped to the joint limits.  A
    free-flyer base starts at a translation U(+-0.5) m with a uniform random orientation and
    moves by U(+-0.2 spread) m and a rotation exp(U(+-0.3 spread)) composed on the right;
    spherical joints likewise in rotation; planar and unbounded joints start at a uniform
    angle and turn by U(+-spread) (planar: translation as the free-flyer's in x, y)."""
    rng = np.random.default_rng(seed)
    lo = model.lower_pos_limit.double().numpy()
    hi = model.upper_pos_limit.double().numpy()
    q0 = rng.uniform(-2.5, 2.5, size=(n, model.nq))
    q1 = np.clip(q0 + rng.uniform(-spread, spread, size=(n, model.nq)), lo, hi)
    q0 = np.clip(q0, lo, hi)
    for j, jm in enumerate(model.joint_models):
        iq = model.idx_qs[j]
        if jm.kind in ("spherical", "planar", "revolute_unbounded"):
            if jm.kind == "spherical":          # unit quaternion, then a rotation exp(U(+-0.3 spread))
                u = rng.normal(size=(n, 4))
                q0[:, iq:iq + 4] = u / np.linalg.norm(u, axis=1, keepdims=True)
                w = rng.uniform(-0.3 * spread, 0.3 * spread, size=(n, 3))
                th = np.linalg.norm(w, axis=1, keepdims=True)
                sh = np.where(th > 1e-12, np.sin(0.5 * th) / np.maximum(th, 1e-12), 0.5)
                q1[:, iq:iq + 4] = _quat_mul_np(q0[:, iq:iq + 4], np.concatenate([sh * w, np.cos(0.5 * th)], 1))
            else:                               # [x, y,] cos, sin of a uniform angle, moved by U(+-spread)
                k = iq + (2 if jm.kind == "planar" else 0)
                th0 = rng.uniform(-np.pi, np.pi, size=n)
                th1 = th0 + rng.uniform(-spread, spread, size=n)
                q0[:, k], q0[:, k + 1] = np.cos(th0), np.sin(th0)
                q1[:, k], q1[:, k + 1] = np.cos(th1), np.sin(th1)
                if jm.kind == "planar":
                    q0[:, iq:iq + 2] = rng.uniform(-0.5, 0.5, size=(n, 2))
                    q1[:, iq:iq + 2] = q0[:, iq:iq + 2] + rng.uniform(-0.2 * spread, 0.2 * spread, size=(n, 2))
            continue
        if jm.kind != "free_flyer":
            continue
        q0[:, iq:iq + 3] = rng.uniform(-0.5, 0.5, size=(n, 3))
        u = rng.normal(size=(n, 4))
        q0[:, iq + 3:iq + 7] = u / np.linalg.norm(u, axis=1, keepdims=True)
        q1[:, iq:iq + 3] = q0[:, iq:iq + 3] + rng.uniform(-0.2 * spread, 0.2 * spread, size=(n, 3))
        w = rng.uniform(-0.3 * spread, 0.3 * spread, size=(n, 3))
        th = np.linalg.norm(w, axis=1, keepdims=True)
        sh = np.where(th > 1e-12, np.sin(0.5 * th) / np.maximum(th, 1e-12), 0.5)
        q1[:, iq + 3:iq + 7] = _quat_mul_np(q0[:, iq + 3:iq + 7], np.concatenate([sh * w, np.cos(0.5 * th)], 1))
    return torch.from_numpy(q0), torch.from_numpy(q1)


def ik_uneven_mix(n_problems: int, seed: int = 3) -> list[tuple[str, int]]:
    """Class label and target count for each problem of the uneven batch:
    40% chain7, 30% dual_arm, 30% humanoid; 1-6 targets each."""
    rng = np.random.default_rng(seed)
    n_chain = int(round(0.4 * n_problems))
    n_dual = int(round(0.3 * n_problems))
    n_hum = n_problems - n_chain - n_dual
    labels = ["chain7"] * n_chain + ["dual_arm"] * n_dual + ["humanoid"] * n_hum
    perm = rng.permutation(n_problems)
    kt = rng.integers(1, 7, size=n_problems)
    return [(labels[i], int(kt[k])) for k, i in enumerate(perm)]


def deg(x: float) -> float:
    return x * 180.0 / math.pi

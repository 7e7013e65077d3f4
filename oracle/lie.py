"""SE3 / SO3 in float64 numpy, batched over leading axes.

Restates ``src/better_robot/lie/_torch_native_backend.py`` and
``src/better_robot/lie/tangents.py``.  Storage ``[tx,ty,tz,qx,qy,qz,qw]``,
tangent ``[vx,vy,vz,wx,wy,wz]`` (linear first).
"""

from __future__ import annotations

import math

import numpy as np

TAYLOR_THETA2 = 1e-8  # _torch_native_backend.py:26


def hat(v: np.ndarray) -> np.ndarray:
    """Skew matrix, ``_torch_native_backend._hat3:31`` / ``tangents.hat_so3:24``."""
    z = np.zeros_like(v[..., 0])
    return np.stack([np.stack([z, -v[..., 2], v[..., 1]], -1),
                     np.stack([v[..., 2], z, -v[..., 0]], -1),
                     np.stack([-v[..., 1], v[..., 0], z], -1)], -2)


def quat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Hamilton product, ``_quat_mul:44-52``."""
    ax, ay, az, aw = np.moveaxis(a, -1, 0)
    bx, by, bz, bw = np.moveaxis(b, -1, 0)
    return np.stack([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz], -1)


def quat_to_matrix(q: np.ndarray) -> np.ndarray:
    """``_quat_to_matrix:55-69``."""
    qx, qy, qz, qw = np.moveaxis(q, -1, 0)
    xx, yy, zz = qx * qx, qy * qy, qz * qz
    xy, xz, yz = qx * qy, qx * qz, qy * qz
    wx, wy, wz = qw * qx, qw * qy, qw * qz
    return np.stack([np.stack([1 - 2 * (yy + zz), 2 * (xy - wz), 2 * (xz + wy)], -1),
                     np.stack([2 * (xy + wz), 1 - 2 * (xx + zz), 2 * (yz - wx)], -1),
                     np.stack([2 * (xz - wy), 2 * (yz + wx), 1 - 2 * (xx + yy)], -1)], -2)


def so3_act(q: np.ndarray, p: np.ndarray) -> np.ndarray:
    """``p' = p + 2 u x (u x p + w p)``, ``so3_act:186-199``."""
    u = q[..., :3]
    w = q[..., 3:4]
    u, p = np.broadcast_arrays(u, p)
    c1 = np.cross(u, p) + w * p
    return p + 2.0 * np.cross(u, c1)


def so3_inverse(q: np.ndarray) -> np.ndarray:
    return q * np.array([-1.0, -1.0, -1.0, 1.0])


def so3_exp(w: np.ndarray) -> np.ndarray:
    """``so3_exp:144-159``."""
    th2 = np.sum(w * w, -1, keepdims=True)
    th = np.sqrt(np.maximum(th2, 0.0))
    half = th / 2.0
    with np.errstate(divide="ignore", invalid="ignore"):
        full = np.sin(half) / np.maximum(th, 1e-30)
    s = np.where(th2 < TAYLOR_THETA2, 0.5 - th2 / 48.0, full)
    return np.concatenate([s * w, np.cos(half)], -1)


def so3_log(q: np.ndarray) -> np.ndarray:
    """``so3_log:162-183`` (folds ``qw < 0``)."""
    q = np.where(q[..., 3:4] < 0, -q, q)
    u = q[..., :3]
    w = q[..., 3:4]
    s2 = np.sum(u * u, -1, keepdims=True)
    s = np.sqrt(np.maximum(s2, 0.0))
    theta = 2.0 * np.arctan2(s, np.clip(w, -1.0, 1.0))
    full = theta / np.maximum(s, 1e-30)
    factor = np.where(s2 < TAYLOR_THETA2 / 4.0, 2.0 + s2 * (2.0 / 3.0), full)
    return factor * u


def se3_compose(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """``se3_compose:237-246``."""
    a, b = np.broadcast_arrays(a, b)
    t = a[..., :3] + so3_act(a[..., 3:7], b[..., :3])
    q = quat_mul(a[..., 3:7], b[..., 3:7])
    return np.concatenate([t, q], -1)


def se3_inverse(T: np.ndarray) -> np.ndarray:
    """``se3_inverse:249-255``."""
    qi = so3_inverse(T[..., 3:7])
    return np.concatenate([-so3_act(qi, T[..., :3]), qi], -1)


def se3_normalize(T: np.ndarray) -> np.ndarray:
    """``se3_normalize:358-361``."""
    q = T[..., 3:7]
    n = np.maximum(np.linalg.norm(q, axis=-1, keepdims=True), 1e-8)
    return np.concatenate([T[..., :3], q / n], -1)


def se3_exp(xi: np.ndarray) -> np.ndarray:
    """``se3_exp:258-286``."""
    v = xi[..., :3]
    w = xi[..., 3:6]
    th2 = np.sum(w * w, -1, keepdims=True)
    th = np.sqrt(np.maximum(th2, 0.0))
    small = th2 < TAYLOR_THETA2
    with np.errstate(divide="ignore", invalid="ignore"):
        b_full = (1.0 - np.cos(th)) / np.maximum(th2, 1e-30)
        c_full = (th - np.sin(th)) / np.maximum(th * th2, 1e-30)
    b = np.where(small, 0.5 - th2 / 24.0, b_full)
    c = np.where(small, 1.0 / 6.0 - th2 / 120.0, c_full)
    W = hat(w)
    V = np.eye(3) + b[..., None] * W + c[..., None] * (W @ W)
    t = (V @ v[..., None])[..., 0]
    return np.concatenate([t, so3_exp(w)], -1)


def se3_log(T: np.ndarray) -> np.ndarray:
    """``se3_log:289-310``."""
    t = T[..., :3]
    w = so3_log(T[..., 3:7])
    th2 = np.sum(w * w, -1, keepdims=True)
    th = np.sqrt(np.maximum(th2, 0.0))
    small = th2 < TAYLOR_THETA2
    half = th / 2.0
    with np.errstate(divide="ignore", invalid="ignore"):
        cot = np.cos(half) / np.maximum(np.sin(half), 1e-30)
        full = 1.0 / np.maximum(th2, 1e-30) - cot / (2.0 * np.maximum(th, 1e-30))
    coeff = np.where(small, 1.0 / 12.0 + th2 / 720.0, full)
    W = hat(w)
    Vinv = np.eye(3) - 0.5 * W + coeff[..., None] * (W @ W)
    v = (Vinv @ t[..., None])[..., 0]
    return np.concatenate([v, w], -1)


def ad_matrix(xi: np.ndarray) -> np.ndarray:
    """``tangents._ad_matrix:164-178``: ``[[hat(w), hat(v)], [0, hat(w)]]``."""
    V = hat(xi[..., :3])
    W = hat(xi[..., 3:])
    Z = np.zeros_like(W)
    return np.concatenate([np.concatenate([W, V], -1), np.concatenate([Z, W], -1)], -2)


def right_jacobian_se3(xi: np.ndarray, terms: int = 9) -> np.ndarray:
    """Truncated series ``sum_{k<=9} (-1)^k/(k+1)! ad^k``, ``tangents.right_jacobian_se3:184-201``."""
    ad = ad_matrix(xi)
    I6 = np.broadcast_to(np.eye(6), ad.shape)
    res = I6.copy()
    pw = I6.copy()
    for k in range(1, terms + 1):
        pw = pw @ ad
        res = res + ((-1.0) ** k) / math.factorial(k + 1) * pw
    return res


def right_jacobian_inv_se3(xi: np.ndarray) -> np.ndarray:
    """``tangents.right_jacobian_inv_se3:204-207`` (inverse of the truncated series)."""
    return np.linalg.inv(right_jacobian_se3(xi))


def se3_act(T: np.ndarray, p: np.ndarray) -> np.ndarray:
    """``se3_act:313-315``: ``R p + t``."""
    return so3_act(T[..., 3:7], p) + T[..., :3]


def se3_adjoint(T: np.ndarray) -> np.ndarray:
    """``se3_adjoint:318-328``: ``[[R, hat(p) R], [0, R]]``."""
    R = quat_to_matrix(T[..., 3:7])
    Z = np.zeros_like(R)
    return np.concatenate([np.concatenate([R, hat(T[..., :3]) @ R], -1), np.concatenate([Z, R], -1)], -2)


def se3_adjoint_inv(T: np.ndarray) -> np.ndarray:
    """``se3_adjoint_inv:331-342``: ``[[R^T, -R^T hat(p)], [0, R^T]]``."""
    RT = np.swapaxes(quat_to_matrix(T[..., 3:7]), -1, -2)
    Z = np.zeros_like(RT)
    return np.concatenate([np.concatenate([RT, -(RT @ hat(T[..., :3]))], -1), np.concatenate([Z, RT], -1)], -2)


def so3_normalize(q: np.ndarray) -> np.ndarray:
    """``so3_normalize:202-203``: ``q / max(|q|, 1e-8)``."""
    return q / np.maximum(np.linalg.norm(q, axis=-1, keepdims=True), 1e-8)


def so3_from_matrix(R: np.ndarray) -> np.ndarray:
    """Shepperd's method with the reference's branch order, ``_matrix_to_quat:72-125``."""
    m = R
    tr = m[..., 0, 0] + m[..., 1, 1] + m[..., 2, 2]
    s1 = np.sqrt(np.maximum(tr + 1.0, 1e-30)) * 2.0
    s2 = np.sqrt(np.maximum(1.0 + m[..., 0, 0] - m[..., 1, 1] - m[..., 2, 2], 1e-30)) * 2.0
    s3 = np.sqrt(np.maximum(1.0 - m[..., 0, 0] + m[..., 1, 1] - m[..., 2, 2], 1e-30)) * 2.0
    s4 = np.sqrt(np.maximum(1.0 - m[..., 0, 0] - m[..., 1, 1] + m[..., 2, 2], 1e-30)) * 2.0
    a = m[..., 2, 1] - m[..., 1, 2]
    b = m[..., 0, 2] - m[..., 2, 0]
    c = m[..., 1, 0] - m[..., 0, 1]
    d = m[..., 0, 1] + m[..., 1, 0]
    e = m[..., 0, 2] + m[..., 2, 0]
    f = m[..., 1, 2] + m[..., 2, 1]
    q1 = np.stack([a / s1, b / s1, c / s1, 0.25 * s1], -1)
    q2 = np.stack([0.25 * s2, d / s2, e / s2, a / s2], -1)
    q3 = np.stack([d / s3, 0.25 * s3, f / s3, b / s3], -1)
    q4 = np.stack([e / s4, f / s4, 0.25 * s4, c / s4], -1)
    c1 = (tr > 0)[..., None]
    c2 = ((m[..., 0, 0] > m[..., 1, 1]) & (m[..., 0, 0] > m[..., 2, 2]))[..., None]
    c3 = (m[..., 1, 1] > m[..., 2, 2])[..., None]
    q = np.where(c1, q1, np.where(c2, q2, np.where(c3, q3, q4)))
    return q / np.maximum(np.linalg.norm(q, axis=-1, keepdims=True), 1e-12)


def right_jacobian_inv_so3(w: np.ndarray) -> np.ndarray:
    """``tangents.right_jacobian_inv_so3:122-145``: ``I + hat/2 + C hat^2``,
    ``C = 1/theta^2 - (1 + cos theta) / (2 theta sin theta)`` (1/12 + theta^2/720 below theta^2 = 1e-10)."""
    th2 = np.sum(w * w, -1)
    th = np.sqrt(np.maximum(th2, 0.0))
    with np.errstate(divide="ignore", invalid="ignore"):
        full = 1.0 / np.maximum(th2, 1e-30) - (1.0 + np.cos(th)) / np.maximum(2.0 * th * np.sin(th), 1e-30)
    C = np.where(th2 > 1e-10, full, 1.0 / 12.0 + th2 / 720.0)
    H = hat(w)
    return np.eye(3) + 0.5 * H + C[..., None, None] * (H @ H)

"""GPU parity of the batched SE3 / SO3 kernels (``br_lie_op``) against the reference's outputs.

Inputs and float64 outputs come from BetterRobot's torch backend (``tests/golden/lie*.npz``).
Tolerances for the float32 kernels:
* quaternions: rotation angle of q_ref^-1 q <= 2e-6 rad (sign-free: q and -q are one rotation);
* translations, points, tangents, matrices: |x - ref| <= 2e-6 * (1 + |ref|), except
  se3_log / so3_log (5e-6) and their rows within 1e-3 rad of pi, where float32 rounding
  of qw alone moves the result by ~1e-4 relative (1e-3 bound there);
* Jr^-1: |dJ| <= 1e-4 * max|J_ref| per element (the frame-Jacobian tolerance).
"""

import os

import numpy as np
import pytest
import torch

from betterrobot_b200 import lie as dlie
from betterrobot_b200.exceptions import DeviceMismatchError, DtypeMismatchError, ShapeError
from oracle import lie

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _g(name):
    return np.load(os.path.join(GOLDEN, name))


def cu(x):
    return torch.from_numpy(np.ascontiguousarray(x)).float().cuda()


def np64(t):
    if isinstance(t, np.ndarray):
        return t.astype(np.float64)
    return t.detach().cpu().double().numpy()


def assert_close(got, ref, tol=2e-6, name=""):
    got = np64(got)
    err = np.abs(got - ref) / (1.0 + np.abs(ref))
    assert err.max() <= tol, f"{name}: max scaled error {err.max():.3e}"


def assert_quat(got, ref, tol=2e-6, name=""):
    got = np64(got)
    qe = lie.quat_mul(lie.so3_inverse(ref), got)
    ang = np.linalg.norm(lie.so3_log(qe / np.linalg.norm(qe, axis=-1, keepdims=True)), axis=-1)
    assert ang.max() <= tol, f"{name}: rotation error {ang.max():.3e}"
    np.testing.assert_allclose(np.linalg.norm(got, axis=-1), 1.0, atol=1e-6)


def assert_pose(got, ref, name=""):
    got = np64(got)
    assert_close(got[..., :3], ref[..., :3], name=name + ".t")
    assert_quat(got[..., 3:], ref[..., 3:], name=name + ".q")


def test_golden_se3_so3_through_cuda():
    g = _g("lie_ops.npz")
    A, B, P, Au = cu(g["A"]), cu(g["B"]), cu(g["P"]), cu(g["A_unnorm"])
    q, qb = A[:, 3:].contiguous(), B[:, 3:].contiguous()
    assert_pose(dlie.se3_compose(A, B), g["se3_compose"], "se3_compose")
    assert_pose(dlie.se3_inverse(A), g["se3_inverse"], "se3_inverse")
    assert_close(dlie.se3_act(A, P), g["se3_act"], name="se3_act")
    assert_close(dlie.se3_adjoint(A), g["se3_adjoint"], name="se3_adjoint")
    assert_close(dlie.se3_adjoint_inv(A), g["se3_adjoint_inv"], name="se3_adjoint_inv")
    assert_pose(dlie.se3_normalize(Au), g["se3_normalize"], "se3_normalize")
    assert_quat(dlie.so3_compose(q, qb), g["so3_compose"], name="so3_compose")
    assert_quat(dlie.so3_inverse(q), g["so3_inverse"], name="so3_inverse")
    assert_close(dlie.so3_act(q, P), g["so3_act"], name="so3_act")
    assert_close(dlie.so3_to_matrix(q), g["so3_to_matrix"], name="so3_to_matrix")
    assert_quat(dlie.so3_from_matrix(cu(g["so3_to_matrix"])), g["so3_from_matrix"], name="so3_from_matrix")
    assert_quat(dlie.so3_normalize(Au[:, 3:].contiguous()), g["so3_normalize"], name="so3_normalize")
    assert_close(dlie.right_jacobian_se3(cu(g["xi"])), g["jr"], name="right_jacobian_se3")
    # logs: rows 0..6 sit within 2e-4 rad of pi
    near_pi = np.abs(np.linalg.norm(g["so3_log"], axis=-1) - np.pi) < 1e-3
    for key, got in (("so3_log", dlie.so3_log(q)), ("se3_log", dlie.se3_log(A))):
        ref, got = g[key], np64(got)
        assert_close(got[~near_pi], ref[~near_pi], tol=5e-6, name=key)
        assert_close(got[near_pi], ref[near_pi], tol=1e-3, name=key + " near pi")


def test_golden_exp_log_jr_inv_through_cuda():
    g = _g("lie.npz")
    xi, T = cu(g["xi"]), cu(g["T_in"])
    assert_pose(dlie.se3_exp(xi), g["se3_exp"], "se3_exp")
    assert_quat(dlie.so3_exp(xi[:, 3:].contiguous()), g["so3_exp"], name="so3_exp")
    assert_close(dlie.se3_log(T), g["se3_log"], tol=5e-6, name="se3_log")
    assert_close(dlie.so3_log(T[:, 3:].contiguous()), g["so3_log"], tol=5e-6, name="so3_log")
    J = np64(dlie.right_jacobian_inv_se3(xi))
    scale = np.abs(g["jr_inv"]).max(axis=(-1, -2), keepdims=True)
    assert (np.abs(J - g["jr_inv"]) / scale).max() <= 1e-4


def test_broadcasting_and_shapes():
    rng = np.random.default_rng(5)
    a = lie.se3_exp(rng.normal(size=(3, 6)))
    b = lie.se3_exp(rng.normal(size=(2, 3, 6)))
    got = dlie.se3_compose(cu(a), cu(b))
    assert got.shape == (2, 3, 7)
    assert_pose(got, lie.se3_compose(a, b), "broadcast")
    one = dlie.se3_compose(cu(a[:1]), cu(b))  # a single element broadcast through the kernel (stride 0)
    assert_pose(one, lie.se3_compose(a[:1], b), "broadcast-one")
    p = rng.normal(size=(4, 1, 3))
    act = dlie.se3_act(cu(a), cu(p))
    assert act.shape == (4, 3, 3)
    assert_close(act, lie.se3_act(a, p), name="act broadcast")
    single = dlie.se3_log(cu(a[0]))
    assert single.shape == (6,)
    assert dlie.se3_adjoint(cu(a)).shape == (3, 6, 6)
    assert dlie.so3_from_matrix(cu(lie.quat_to_matrix(a[:, 3:]))).shape == (3, 4)
    empty = dlie.se3_inverse(torch.empty(0, 7, device="cuda"))
    assert empty.shape == (0, 7)


def test_large_batch_grid_stride():
    """2^21 elements: more than one element per thread of the capped grid."""
    n = 1 << 21
    g = torch.Generator(device="cuda").manual_seed(3)
    xi = torch.randn(n, 6, device="cuda", generator=g)
    T = dlie.se3_exp(xi)
    back = dlie.se3_log(T)
    small = xi[:, 3:].norm(dim=-1) < 3.0
    assert float((back[small] - xi[small]).abs().max()) < 5e-5  # exp/log round trip below pi
    idx = torch.randint(0, n, (4096,), device="cuda", generator=g)
    assert_pose(T[idx], lie.se3_exp(np64(xi[idx])), "exp sample")
    I = dlie.se3_compose(T, dlie.se3_inverse(T))
    assert float(I[:, :3].abs().max()) < 1e-4 and float((I[:, 6].abs() - 1).abs().max()) < 1e-6


def test_log_rotation_angle_sweep():
    """The SE3 / SO3 logs' rotation angle over 2^20 angles in [0, pi) and random axes, against
    float64 on the float32 inputs: within 2e-6 rad (about 8 ulp of pi; the SE3 log's fitted
    first-quadrant arctangent and its square root / reciprocal estimates measured 1.05e-6 at
    worst, near pi), inside the 5e-6 scaled bound of the logs above."""
    n = 1 << 20
    rng = np.random.default_rng(22)
    th = np.linspace(0.0, np.pi, n, endpoint=False)
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    q = np.concatenate([np.sin(th / 2)[:, None] * ax, np.cos(th / 2)[:, None]], axis=1)
    T = np.concatenate([rng.normal(size=(n, 3)), q], axis=1)
    Tc = cu(T)
    q32 = np64(Tc[:, 3:])
    exact = 2.0 * np.arctan2(np.linalg.norm(q32[:, :3], axis=1), np.abs(q32[:, 3]))
    got = np.linalg.norm(np64(dlie.se3_log(Tc))[:, 3:], axis=1)
    assert np.abs(got - exact).max() <= 2e-6, np.abs(got - exact).max()
    got = np.linalg.norm(np64(dlie.so3_log(Tc[:, 3:].contiguous())), axis=1)
    assert np.abs(got - exact).max() <= 2e-6, np.abs(got - exact).max()
    # the translation part against the float64 oracle on a sample
    idx = rng.choice(n, 4096, replace=False)
    assert_close(dlie.se3_log(Tc[idx]), lie.se3_log(np64(Tc[idx])), tol=5e-6, name="se3_log sweep")


def test_wide_outputs_large_batch():
    """2^18 elements through the ops with 36-float outputs (SE3 adjoint / adjoint-inverse stage
    one input buffer per warp, Jr / Jr^-1 two): every warp of every CTA busy, grid-stride, a
    ragged last tile; every row against the float64 oracle."""
    n = (1 << 18) + 7
    rng = np.random.default_rng(21)
    T = rng.normal(size=(n, 7))
    T[:, 3:] /= np.linalg.norm(T[:, 3:], axis=1, keepdims=True)
    Tc = cu(T)
    assert_close(dlie.se3_adjoint(Tc).reshape(n, 36), lie.se3_adjoint(np64(Tc)).reshape(n, 36), name="se3_adjoint")
    assert_close(dlie.se3_adjoint_inv(Tc).reshape(n, 36), lie.se3_adjoint_inv(np64(Tc)).reshape(n, 36),
                 name="se3_adjoint_inv")
    xi = cu(rng.normal(scale=0.5, size=(n, 6)))
    Jr = dlie.right_jacobian_se3(xi).reshape(n, 36)
    ref = lie.right_jacobian_se3(np64(xi)).reshape(n, 36)
    assert_close(Jr, ref, tol=1e-5, name="right_jacobian_se3")


def test_boundary_errors():
    with pytest.raises(DeviceMismatchError):
        dlie.se3_log(torch.zeros(2, 7))
    with pytest.raises(DtypeMismatchError):
        dlie.se3_log(torch.zeros(2, 7, device="cuda", dtype=torch.float64))
    with pytest.raises(ShapeError):
        dlie.se3_log(torch.zeros(2, 6, device="cuda"))
    with pytest.raises(ShapeError):
        dlie.so3_from_matrix(torch.zeros(2, 9, device="cuda"))
    with pytest.raises(RuntimeError):
        dlie.se3_compose(torch.zeros(2, 7, device="cuda"), torch.zeros(3, 7, device="cuda"))

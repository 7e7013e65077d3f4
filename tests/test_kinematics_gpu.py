"""GPU parity of FK / frame Jacobians against the float64 oracle.

Tolerances (float32 kernel vs float64 oracle):
* positions: max |dp| <= 1e-5 m;
* rotations: angle of q_ref^-1 q <= 1e-5 rad;
* Jacobians: |dJ| <= 1e-4 * max|J_ref| of the same (configuration, frame) block.
"""

import os

import numpy as np
import pytest
import torch

import betterrobot_b200 as br
from betterrobot_b200 import synthetic as syn
from oracle import kinematics as K, lie

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
ROT_TOL = 1e-5
JAC_TOL = 1e-4
SPECS = {"chain7": syn.chain_spec(), "humanoid": syn.humanoid_spec(), "dual_arm": syn.dual_arm_spec(),
         "mixed": syn.mixed_spec()}  # mixed: planar base, translation, spherical and unbounded joints


def assert_poses(got, ref):
    got = got.detach().cpu().double().numpy().reshape(-1, 7)
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, 7)
    dp = np.abs(got[:, :3] - ref[:, :3]).max()
    qe = lie.quat_mul(lie.so3_inverse(ref[:, 3:]), got[:, 3:])
    ang = np.linalg.norm(lie.so3_log(qe / np.linalg.norm(qe, axis=-1, keepdims=True)), axis=-1).max()
    assert dp <= POS_TOL, f"position error {dp:.3e}"
    assert ang <= ROT_TOL, f"rotation error {ang:.3e}"


def assert_jac(got, ref):
    got = got.detach().cpu().double().numpy()
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.abs(ref).max(axis=(-1, -2), keepdims=True)
    err = (np.abs(got - ref) / np.maximum(scale, 1e-12)).max()
    assert err <= JAC_TOL, f"relative Jacobian error {err:.3e}"


@pytest.fixture(scope="module", params=list(SPECS))
def robot(request):
    name = request.param
    return name, syn.model_from_spec(SPECS[name]), syn.model_from_spec(SPECS[name], dtype=torch.float64)


@pytest.mark.parametrize("B", [1, 5, 33, 1000])
def test_forward_kinematics_matches_oracle(robot, B):
    name, m, m64 = robot
    q = syn.random_q(m64, B, 100 + B, rev_range=2.5, base_translation=1.0)
    data = br.forward_kinematics(m, q.float().cuda(), compute_frames=True)
    oMi, liMi = K.forward_kinematics(m64, q.numpy())
    assert data.joint_pose_world.shape == (B, m.njoints, 7)
    assert_poses(data.joint_pose_world, oMi)
    assert_poses(data.joint_pose_local, liMi)
    assert_poses(data.frame_pose_world, K.frame_placements(m64, oMi))


@pytest.mark.parametrize("name", list(SPECS))
def test_golden_fixture_through_cuda(name):
    """The reference's own float64 outputs (golden) reproduced by the CUDA path."""
    g = np.load(os.path.join(GOLDEN, f"kin_{name}.npz"))
    m = syn.model_from_spec(SPECS[name])
    q = torch.from_numpy(g["q"]).float().cuda()
    data = br.forward_kinematics(m, q, compute_frames=True)
    assert_poses(data.joint_pose_world, g["oMi"])
    assert_poses(data.frame_pose_world, g["oMf"])
    fids = [int(f) for f in g["frame_ids"]]
    for ref, key in (("world", "J_world"), ("local_world_aligned", "J_lwa"), ("local", "J_local")):
        _, J = br.frame_jacobians(m, q, fids, reference=ref)
        assert_jac(J, g[key])
        J1 = br.get_frame_jacobian(m, data, fids[0], reference=ref)
        assert_jac(J1, g[key][:, 0])
    br.compute_joint_jacobians(m, data)
    assert_jac(data.joint_jacobians, g["joint_jacobians"])
    from betterrobot_b200.configuration import difference, integrate
    np.testing.assert_allclose(integrate(m, q, torch.from_numpy(g["v"]).float().cuda()).cpu().double().numpy(),
                               g["integrate"], atol=2e-6, rtol=0)
    np.testing.assert_allclose(difference(m, q, torch.from_numpy(g["q1"]).float().cuda()).cpu().double().numpy(),
                               g["difference"], atol=2e-6, rtol=0)


@pytest.mark.parametrize("reference", ["world", "local_world_aligned", "local"])
@pytest.mark.parametrize("B", [1, 31, 257])
def test_frame_jacobians_match_oracle(robot, reference, B):
    name, m, m64 = robot
    q = syn.random_q(m64, B, 7 + B, rev_range=2.5, base_translation=1.0)
    fids = list(range(m.nframes))[-min(12, m.nframes):]
    T, J = br.frame_jacobians(m, q.float().cuda(), fids, reference=reference)
    oMi, _ = K.forward_kinematics(m64, q.numpy())
    assert_poses(T, K.frame_placements(m64, oMi, fids))
    Jref = np.stack([K.frame_jacobian(m64, oMi, q.numpy(), f, reference) for f in fids], -3)
    assert_jac(J, Jref)


@pytest.mark.parametrize("reference", ["world", "local_world_aligned", "local"])
def test_large_jacobian_blocks_match_oracle(reference):
    """Every frame of the humanoid (44: a 38 KB Jacobian block per configuration, staged and
    stored in pieces of eight targets), and all 32 joints from stored placements
    (compute_joint_jacobians, 27.6 KB blocks), against the oracle; B = 129 leaves partial CTAs."""
    m = syn.model_from_spec(SPECS["humanoid"])
    m64 = syn.model_from_spec(SPECS["humanoid"], dtype=torch.float64)
    q = syn.random_q(m64, 129, 91, rev_range=2.5, base_translation=1.0)
    fids = list(range(m.nframes))
    T, J = br.frame_jacobians(m, q.float().cuda(), fids, reference=reference)
    oMi, _ = K.forward_kinematics(m64, q.numpy())
    assert_poses(T, K.frame_placements(m64, oMi, fids))
    assert_jac(J, np.stack([K.frame_jacobian(m64, oMi, q.numpy(), f, reference) for f in fids], -3))
    if reference == "world":
        data = br.compute_joint_jacobians(m, br.forward_kinematics(m, q.float().cuda()))
        assert_jac(data.joint_jacobians, K.compute_joint_jacobians(m64, oMi, q.numpy()))


@pytest.mark.parametrize("reference", ["world", "local_world_aligned", "local"])
def test_large_unaligned_jacobian_blocks_in_pieces(reference):
    """A 33-DOF chain with 21 body frames: a 16.6 KB J block per configuration, staged in pieces
    of ten targets (10, 10, 1), whose 7,920 B pieces and 16,632 B block are stored lane by lane
    (21 x 33 is odd: the block is not a multiple of 16 bytes); B = 70 leaves partial CTAs."""
    spec = syn.chain_spec(seed=12, n=33, name="chain33")
    m = syn.model_from_spec(spec)
    m64 = syn.model_from_spec(spec, dtype=torch.float64)
    fids = [m.frame_id(f"body_link{i}") for i in (*range(3, 34, 3), *range(1, 31, 3))]
    assert len(fids) == 21
    q = syn.random_q(m64, 70, 17)
    T, J = br.frame_jacobians(m, q.float().cuda(), fids, reference=reference)
    oMi, _ = K.forward_kinematics(m64, q.numpy())
    assert_poses(T, K.frame_placements(m64, oMi, fids))
    assert_jac(J, np.stack([K.frame_jacobian(m64, oMi, q.numpy(), f, reference) for f in fids], -3))


def test_unaligned_output_fallback_chain():
    """chain7 with one frame: a J block is 168 B (not a multiple of 16) -> cooperative stores."""
    m = syn.model_from_spec(SPECS["chain7"])
    m64 = syn.model_from_spec(SPECS["chain7"], dtype=torch.float64)
    q = syn.random_q(m64, 77, 3)
    fid = m.frame_id("ee")
    T, J = br.frame_jacobians(m, q.float().cuda(), [fid])
    oMi, _ = K.forward_kinematics(m64, q.numpy())
    assert_jac(J, K.frame_jacobian(m64, oMi, q.numpy(), fid)[:, None])
    assert_poses(T, K.frame_placements(m64, oMi, [fid]))


def test_humanoid_full_batch_properties():
    """Config-1 size (B=65,536, 12 frames): sampled parity + unit quaternions + determinism."""
    m = syn.model_from_spec(SPECS["humanoid"])
    m64 = syn.model_from_spec(SPECS["humanoid"], dtype=torch.float64)
    fids = syn.op_frame_ids(m)
    q = syn.random_q(m64, 65536, 1, rev_range=2.5, base_translation=1.0)
    qc = q.float().cuda()
    T, J = br.frame_jacobians(m, qc, fids)
    T2, J2 = br.frame_jacobians(m, qc, fids)
    assert torch.equal(J, J2) and torch.equal(T, T2)
    assert J.shape == (65536, 12, 6, m.nv)
    qn = T[..., 3:].norm(dim=-1)
    assert float((qn - 1).abs().max()) < 1e-5
    idx = np.random.default_rng(0).choice(65536, 512, replace=False)
    oMi, _ = K.forward_kinematics(m64, q.numpy()[idx])
    assert_poses(T[idx], K.frame_placements(m64, oMi, fids))
    Jref = np.stack([K.frame_jacobian(m64, oMi, q.numpy()[idx], f) for f in fids], -3)
    assert_jac(J[idx], Jref)


def test_unbatched_and_multi_batch_dims():
    name, m = "dual_arm", syn.model_from_spec(SPECS["dual_arm"])
    m64 = syn.model_from_spec(SPECS["dual_arm"], dtype=torch.float64)
    q = syn.random_q(m64, 6, 9)
    d1 = br.forward_kinematics(m, q[0].float().cuda())
    assert d1.joint_pose_world.shape == (m.njoints, 7)
    d2 = br.forward_kinematics(m, q.reshape(2, 3, -1).float().cuda())
    assert d2.joint_pose_world.shape == (2, 3, m.njoints, 7)
    oMi, _ = K.forward_kinematics(m64, q.numpy())
    assert_poses(d2.joint_pose_world.reshape(6, -1, 7), oMi)


def test_boundary_errors():
    m = syn.model_from_spec(SPECS["humanoid"])
    q = torch.zeros(4, m.nq, device="cuda")
    with pytest.raises(br.QuaternionNormError):
        br.forward_kinematics(m, q)
    with pytest.raises(br.ShapeError):
        br.forward_kinematics(m, torch.zeros(4, m.nq - 1, device="cuda"))
    with pytest.raises(br.DtypeMismatchError):
        br.forward_kinematics(m, torch.zeros(4, m.nq, device="cuda", dtype=torch.float64))
    data = br.Data(q=torch.zeros(2, m.nq, device="cuda"))
    with pytest.raises(br.StaleCacheError):
        br.get_frame_jacobian(m, data, 0)
    with pytest.raises(ValueError):
        d = br.forward_kinematics(m, torch.tensor([[0, 0, 0, 0, 0, 0, 1.0] + [0.0] * 30], device="cuda"))
        br.get_frame_jacobian(m, d, 0, reference="bogus")


@pytest.mark.parametrize("name,B", [("humanoid", 300), ("dual_arm", 300), ("chain7", 45), ("humanoid", 1),
                                    ("mixed", 300)])
def test_integrate_difference_match_oracle(name, B):
    """B = 300 / 45 leave a ragged last tile of 32 configurations; chain7 has no free-flyer."""
    from betterrobot_b200.configuration import difference, integrate
    m = syn.model_from_spec(SPECS[name])
    m64 = syn.model_from_spec(SPECS[name], dtype=torch.float64)
    q = syn.random_q(m64, B, 5, rev_range=2.5, base_translation=1.0)
    v = torch.from_numpy(np.random.default_rng(6).normal(0, 0.4, size=(B, m.nv)))
    q1 = syn.noisy_start(m64, q, 0.3, 7)
    qi = integrate(m, q.float().cuda(), v.float().cuda())
    ref = K.integrate(m64, q.float().double().numpy(), v.float().double().numpy())
    np.testing.assert_allclose(qi.cpu().double().numpy(), ref, atol=2e-6, rtol=0)
    dv = difference(m, q.float().cuda(), q1.float().cuda())
    ref = K.difference(m64, q.float().double().numpy(), q1.float().double().numpy())
    np.testing.assert_allclose(dv.cpu().double().numpy(), ref, atol=2e-6, rtol=0)
    # round trip: q (+) (q1 (-) q) == q1
    back = integrate(m, q.float().cuda(), dv)
    np.testing.assert_allclose(back.cpu().double().numpy(), q1.float().double().numpy(), atol=1e-5, rtol=0)


def test_integrate_difference_large_batch_round_trip():
    """2^20 humanoid configurations (grid-stride over 32-configuration tiles): q (+) (q1 (-) q) == q1."""
    from betterrobot_b200.configuration import difference, integrate
    m = syn.model_from_spec(SPECS["humanoid"])
    m64 = syn.model_from_spec(SPECS["humanoid"], dtype=torch.float64)
    B = 1 << 20
    q = syn.random_q(m64, B, 11, rev_range=2.5, base_translation=1.0).float().cuda()
    q1 = syn.noisy_start(m64, q[:4096].double().cpu(), 0.3, 12).float().cuda().repeat(B // 4096, 1)
    dv = difference(m, q, q1)
    back = integrate(m, q, dv)
    # quaternion slots compared up to sign; translation and revolute slots directly
    err_t = (back[:, :3] - q1[:, :3]).abs().max()
    dq = torch.minimum((back[:, 3:7] - q1[:, 3:7]).abs().amax(-1), (back[:, 3:7] + q1[:, 3:7]).abs().amax(-1))
    err_r = (back[:, 7:] - q1[:, 7:]).abs().max()
    assert float(err_t) < 2e-5 and float(dq.max()) < 2e-5 and float(err_r) < 2e-5
    idx = np.random.default_rng(13).choice(B, 256, replace=False)
    ref = K.difference(m64, q[idx].double().cpu().numpy(), q1[idx].double().cpu().numpy())
    np.testing.assert_allclose(dv[idx].cpu().double().numpy(), ref, atol=2e-6, rtol=0)


def test_integrate_difference_unaligned_pointers_match():
    """Inputs / outputs that start 4 bytes past a 16-byte boundary take the 4-byte load path: same results."""
    from betterrobot_b200.configuration import difference_into, integrate_into
    m = syn.model_from_spec(SPECS["humanoid"])
    m64 = syn.model_from_spec(SPECS["humanoid"], dtype=torch.float64)
    B = 1000
    q = syn.random_q(m64, B, 21, rev_range=2.5, base_translation=1.0).float().cuda()
    q1 = syn.noisy_start(m64, q.double().cpu(), 0.3, 22).float().cuda()
    v = torch.randn(B, m.nv, device="cuda", generator=torch.Generator("cuda").manual_seed(23)) * 0.3

    def shifted(t):
        buf = torch.empty(t.numel() + 1, device="cuda")[1:].view(t.shape)
        buf.copy_(t)
        assert buf.data_ptr() % 16 != 0
        return buf
    ref_q, ref_v = torch.empty_like(q), torch.empty_like(v)
    integrate_into(m, q, v, ref_q)
    difference_into(m, q, q1, ref_v)
    out_q, out_v = shifted(torch.zeros_like(q)), shifted(torch.zeros_like(v))
    integrate_into(m, shifted(q), shifted(v), out_q)
    difference_into(m, shifted(q), shifted(q1), out_v)
    assert torch.equal(out_q, ref_q) and torch.equal(out_v, ref_v)


def test_empty_batches():
    """B = 0 everywhere: outputs of shape (0, ...) and no launch."""
    m = syn.model_from_spec(SPECS["humanoid"])
    q = torch.zeros(0, m.nq, device="cuda")
    data = br.forward_kinematics(m, q, compute_frames=True)
    assert data.joint_pose_world.shape == (0, m.njoints, 7)
    assert data.frame_pose_world.shape[0] == 0
    fids = syn.op_frame_ids(m)
    T, J = br.frame_jacobians(m, q, fids)
    assert T.shape == (0, len(fids), 7) and J.shape == (0, len(fids), 6, m.nv)
    br.compute_joint_jacobians(m, data)
    assert data.joint_jacobians.shape == (0, m.njoints, 6, m.nv)
    from betterrobot_b200.configuration import difference, integrate
    assert integrate(m, q, torch.zeros(0, m.nv, device="cuda")).shape == (0, m.nq)
    assert difference(m, q, q).shape == (0, m.nv)

"""The ``Backend`` bundle (kinematics + Lie ops) and ``graph_capture`` on the GPU.

Tolerances as in the kinematics tests: positions 1e-5 m, rotations 1e-5 rad, Jacobians
1e-4 relative to the largest entry of each block.
"""

import os

import numpy as np
import pytest
import torch

from betterrobot_b200 import synthetic as syn
from betterrobot_b200.backend import BACKEND, B200Backend, graph_capture
from betterrobot_b200.exceptions import BackendNotAvailableError
from betterrobot_b200.kinematics import frame_jacobians
from oracle import kinematics as K, lie

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

# Method names of the reference's Protocols (src/better_robot/backends/protocol.py:27-110).
LIE_METHODS = ["se3_compose", "se3_inverse", "se3_log", "se3_exp", "se3_act", "se3_adjoint", "se3_adjoint_inv",
               "se3_normalize", "so3_compose", "so3_inverse", "so3_log", "so3_exp", "so3_act", "so3_to_matrix",
               "so3_from_matrix", "so3_normalize"]
KIN_METHODS = ["forward_kinematics", "compute_joint_jacobians"]
DYN_METHODS = ["rnea", "aba", "crba", "center_of_mass"]


def test_bundle_has_protocol_surface():
    assert BACKEND.name == "b200"
    for names, ops in ((LIE_METHODS, BACKEND.lie), (KIN_METHODS, BACKEND.kinematics),
                       (DYN_METHODS, BACKEND.dynamics)):
        for n in names:
            assert callable(getattr(ops, n)), n
    with pytest.raises(BackendNotAvailableError):
        BACKEND.dynamics.rnea(None, None, None, None, None)
    sentinel = object()
    assert B200Backend(dynamics=sentinel).dynamics is sentinel


@pytest.mark.parametrize("name", ["humanoid", "dual_arm"])
def test_kinematics_ops_match_golden(name):
    g = np.load(os.path.join(GOLDEN, f"kin_{name}.npz"))
    spec = syn.humanoid_spec() if name == "humanoid" else syn.dual_arm_spec()
    m = syn.model_from_spec(spec)
    q = torch.from_numpy(g["q"]).float().cuda()
    oMi, liMi = BACKEND.kinematics.forward_kinematics(m, q)
    for got, ref in ((oMi, g["oMi"]), (liMi, g["liMi"])):
        got = got.cpu().double().numpy()
        assert np.abs(got[..., :3] - ref[..., :3]).max() <= 1e-5
        qe = lie.quat_mul(lie.so3_inverse(ref[..., 3:]), got[..., 3:])
        assert np.linalg.norm(lie.so3_log(qe / np.linalg.norm(qe, axis=-1, keepdims=True)), axis=-1).max() <= 1e-5

    class RefData:  # only the attribute the protocol reads
        joint_pose_world = oMi
    J = BACKEND.kinematics.compute_joint_jacobians(m, RefData()).cpu().double().numpy()
    ref = g["joint_jacobians"]
    scale = np.maximum(np.abs(ref).max(axis=(-1, -2), keepdims=True), 1e-12)
    assert (np.abs(J - ref) / scale).max() <= 1e-4
    with pytest.raises(BackendNotAvailableError):
        BACKEND.kinematics.forward_kinematics(m, q.clone().requires_grad_(True))


def test_lie_ops_through_bundle():
    rng = np.random.default_rng(8)
    a = lie.se3_exp(rng.normal(size=(50, 6)))
    b = lie.se3_exp(rng.normal(size=(50, 6)))
    c = BACKEND.lie.se3_compose(torch.from_numpy(a).float().cuda(), torch.from_numpy(b).float().cuda())
    ref = lie.se3_compose(a, b)
    assert np.abs(c.cpu().double().numpy()[:, :3] - ref[:, :3]).max() < 1e-5
    w = BACKEND.lie.se3_log(c).cpu().double().numpy()
    assert np.abs(w - lie.se3_log(ref)).max() < 5e-5


def test_graph_capture_replays_fused_path():
    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    fids = syn.op_frame_ids(m)

    @graph_capture
    def step(q):
        T, J = frame_jacobians(m, q, fids)
        return BACKEND.lie.se3_log(T), J

    outs = []
    for seed in (1, 2, 3):
        q = syn.random_q(m64, 512, seed, rev_range=2.5, base_translation=1.0).float().cuda()
        log, J = step(q)
        T2, J2 = frame_jacobians(m, q, fids)
        assert torch.equal(J, J2)
        assert torch.equal(log, BACKEND.lie.se3_log(T2))
        outs.append(J.clone())
        qn = q.double().cpu().numpy()[:8]
        oMi, _ = K.forward_kinematics(m64, qn)
        Jref = np.stack([K.frame_jacobian(m64, oMi, qn, f) for f in fids], -3)
        scale = np.abs(Jref).max(axis=(-1, -2), keepdims=True)
        assert (np.abs(J[:8].cpu().double().numpy() - Jref) / scale).max() <= 1e-4
    assert len(step.graphs) == 1  # one signature, one graph, replayed for seeds 2 and 3
    assert not torch.equal(outs[0], outs[1])

"""``torch.ops.br_cuda.*`` registration and shape rules, on the CPU (fake tensors: no kernel runs)."""

import torch
from torch._subclasses.fake_tensor import FakeTensorMode

from betterrobot_b200 import synthetic as syn
from betterrobot_b200 import torch_ops

OPS = ["forward_kinematics", "frame_jacobians", "joint_jacobians", "integrate", "difference", "lie_op",
       "pose_loss", "pose_loss_backward"]


def test_operators_registered():
    for name in OPS:
        assert hasattr(torch.ops.br_cuda, name), name


def test_fake_shapes():
    m = syn.model_from_spec(syn.humanoid_spec())
    h = torch_ops.register_model(m)
    with FakeTensorMode():
        q = torch.empty(4, 3, m.nq, device="cuda")
        T, J = torch.ops.br_cuda.frame_jacobians(q, h, [1, 2, 3], 1)
        assert T.shape == (4, 3, 3, 7) and J.shape == (4, 3, 3, 6, m.nv)
        w, loc = torch.ops.br_cuda.forward_kinematics(q, h)
        assert w.shape == loc.shape == (4, 3, m.njoints, 7)
        assert torch.ops.br_cuda.joint_jacobians(w, h).shape == (4, 3, m.njoints, 6, m.nv)
        assert torch.ops.br_cuda.integrate(q, torch.empty(4, 3, m.nv, device="cuda"), h).shape == q.shape
        assert torch.ops.br_cuda.difference(q, q, h).shape == (4, 3, m.nv)
        assert torch.ops.br_cuda.lie_op("se3_adjoint", torch.empty(5, 7, device="cuda")).shape == (5, 6, 6)
        assert torch.ops.br_cuda.lie_op("so3_from_matrix", torch.empty(5, 3, 3, device="cuda")).shape == (5, 4)
        q2 = torch.empty(6, m.nq, device="cuda")
        loss = torch.ops.br_cuda.pose_loss(q2, h, [1, 2], torch.empty(6, 2, 7, device="cuda"),
                                           torch.empty(2, device="cuda"))
        assert loss.shape == (6,)

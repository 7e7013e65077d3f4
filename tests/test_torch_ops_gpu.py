"""``torch.ops.br_cuda.*`` on the GPU: same results as the Python entry points, operator checks,
a full-graph ``torch.compile`` trace, and gradients through the registered adjoint."""

import numpy as np
import pytest
import torch

from betterrobot_b200 import synthetic as syn
from betterrobot_b200 import torch_ops
from betterrobot_b200.adjoint import pose_loss
from betterrobot_b200.kinematics import frame_jacobians

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def humanoid():
    m = syn.model_from_spec(syn.humanoid_spec())
    m64 = syn.model_from_spec(syn.humanoid_spec(), dtype=torch.float64)
    q = syn.random_q(m64, 256, 4, rev_range=2.5, base_translation=1.0).float().cuda()
    return m, torch_ops.register_model(m), q


def test_ops_match_python_api(humanoid):
    m, h, q = humanoid
    fids = syn.op_frame_ids(m)
    T, J = torch.ops.br_cuda.frame_jacobians(q, h, fids, 1)
    T2, J2 = frame_jacobians(m, q, fids)
    assert torch.equal(T, T2) and torch.equal(J, J2)
    w, _ = torch.ops.br_cuda.forward_kinematics(q, h)
    Jj = torch.ops.br_cuda.joint_jacobians(w, h)
    assert Jj.shape == (256, m.njoints, 6, m.nv)
    v = torch.randn(256, m.nv, device="cuda") * 0.1
    q1 = torch.ops.br_cuda.integrate(q, v, h)
    dv = torch.ops.br_cuda.difference(q, q1, h)
    assert float((dv - v).abs().max()) < 1e-4
    log = torch.ops.br_cuda.lie_op("se3_log", T)
    assert log.shape == (256, len(fids), 6)


def test_opcheck(humanoid):
    m, h, q = humanoid
    fids = syn.op_frame_ids(m)[:4]
    torch.library.opcheck(torch.ops.br_cuda.frame_jacobians.default, (q[:32], h, fids, 1),
                          test_utils=("test_schema", "test_faketensor"))
    torch.library.opcheck(torch.ops.br_cuda.lie_op.default, ("se3_exp", torch.randn(16, 6, device="cuda")),
                          test_utils=("test_schema", "test_faketensor"))


def test_compile_fullgraph_and_adjoint_gradient(humanoid):
    m, h, q = humanoid
    fids = syn.op_frame_ids(m)
    B = q.shape[0]
    targets = syn.random_targets(B, len(fids), 5).float().cuda()
    w = torch.from_numpy(np.random.default_rng(6).uniform(0.5, 2.0, size=len(fids))).float().cuda()

    def f(q):
        T, J = torch.ops.br_cuda.frame_jacobians(q.detach(), h, fids, 1)  # FK / J: no autograd formula
        loss = torch.ops.br_cuda.pose_loss(q, h, fids, targets, w)       # differentiable: the adjoint
        return loss.sum(), T, J

    compiled = torch.compile(f, backend="aot_eager", fullgraph=True)
    qa = q.clone().requires_grad_(True)
    out, T, J = compiled(qa)
    out.backward()
    T2, J2 = frame_jacobians(m, q, fids)
    assert torch.equal(T, T2) and torch.equal(J, J2)
    qb = q.clone().requires_grad_(True)
    ref = pose_loss(m, qb, fids, targets, w, mode="recompute").sum()
    ref.backward()
    assert torch.allclose(out, ref, rtol=1e-6, atol=0)
    assert torch.allclose(qa.grad, qb.grad, rtol=1e-5, atol=1e-6)

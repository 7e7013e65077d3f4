"""``torch.ops.br_cuda.*``: the kernels as registered PyTorch custom operators.

Registering them (``torch.library.custom_op`` with a fake implementation that only
computes output shapes) lets ``torch.compile`` and other tracers treat each kernel as
one opaque node instead of graph-breaking on a ctypes call, and lets autograd route
``pose_loss`` through the hand-written adjoint.  Operators take a model *handle*
(``register_model(model) -> int``) because an operator schema holds tensors and
scalars only.

    h = register_model(model)
    T, J = torch.ops.br_cuda.frame_jacobians(q, h, frame_ids, 1)   # 1 = local_world_aligned
"""

from __future__ import annotations

from typing import Sequence

import torch

from . import configuration as _cfg
from . import kinematics as _kin
from . import lie as _lie
from .exceptions import ShapeError

_MODELS: dict[int, object] = {}


def register_model(model) -> int:
    """Handle for ``model`` in the ``br_cuda`` operators (the model object stays referenced)."""
    h = id(model)
    _MODELS[h] = model
    return h


def _model(h: int):
    try:
        return _MODELS[int(h)]
    except KeyError:
        raise ShapeError(f"unknown model handle {h}; call register_model(model) first") from None


_REFS = ("world", "local_world_aligned", "local")


@torch.library.custom_op("br_cuda::forward_kinematics", mutates_args=())
def forward_kinematics(q: torch.Tensor, model: int) -> tuple[torch.Tensor, torch.Tensor]:
    """``(joint_pose_world, joint_pose_local)``, each ``(B..., njoints, 7)``."""
    d = _kin.forward_kinematics(_model(model), q, check_quaternion=False)
    return d.joint_pose_world, d.joint_pose_local


@forward_kinematics.register_fake
def _(q, model):
    m = _model(model)
    shape = (*q.shape[:-1], m.njoints, 7)
    return q.new_empty(shape), q.new_empty(shape)


@torch.library.custom_op("br_cuda::frame_jacobians", mutates_args=())
def frame_jacobians(q: torch.Tensor, model: int, frame_ids: Sequence[int], reference: int
                    ) -> tuple[torch.Tensor, torch.Tensor]:
    """Fused FK + frame Jacobians: ``(oMf (B..., F, 7), J (B..., F, 6, nv))``; reference 0/1/2."""
    T, J = _kin.frame_jacobians(_model(model), q, list(frame_ids), reference=_REFS[reference])
    return T, J


@frame_jacobians.register_fake
def _(q, model, frame_ids, reference):
    m = _model(model)
    F = len(frame_ids)
    return q.new_empty((*q.shape[:-1], F, 7)), q.new_empty((*q.shape[:-1], F, 6, m.nv))


@torch.library.custom_op("br_cuda::joint_jacobians", mutates_args=())
def joint_jacobians(joint_pose_world: torch.Tensor, model: int) -> torch.Tensor:
    """World joint Jacobians ``(B..., njoints, 6, nv)`` from ``joint_pose_world``."""
    m = _model(model)

    class _D:
        pass
    d = _D()
    d.joint_pose_world = joint_pose_world
    return _kin._jac_from_poses(m, d, [-(j + 1) for j in range(m.njoints)], "world")


@joint_jacobians.register_fake
def _(joint_pose_world, model):
    m = _model(model)
    return joint_pose_world.new_empty((*joint_pose_world.shape[:-2], m.njoints, 6, m.nv))


@torch.library.custom_op("br_cuda::integrate", mutates_args=())
def integrate(q: torch.Tensor, v: torch.Tensor, model: int) -> torch.Tensor:
    """``Model.integrate``: ``q (+) v``."""
    return _cfg.integrate(_model(model), q, v)


@integrate.register_fake
def _(q, v, model):
    return q.new_empty((*torch.broadcast_shapes(q.shape[:-1], v.shape[:-1]), q.shape[-1]))


@torch.library.custom_op("br_cuda::difference", mutates_args=())
def difference(q0: torch.Tensor, q1: torch.Tensor, model: int) -> torch.Tensor:
    """``Model.difference``: ``q1 (-) q0``."""
    return _cfg.difference(_model(model), q0, q1)


@difference.register_fake
def _(q0, q1, model):
    return q0.new_empty((*torch.broadcast_shapes(q0.shape[:-1], q1.shape[:-1]), _model(model).nv))


@torch.library.custom_op("br_cuda::lie_op", mutates_args=())
def lie_op(name: str, a: torch.Tensor, b: torch.Tensor | None = None) -> torch.Tensor:
    """Batched SE3 / SO3 op ``name`` (``betterrobot_b200.lie.OPS``)."""
    return _lie.apply(name, a, b)


@lie_op.register_fake
def _(name, a, b=None):
    na, nb, no = _lie._sizes(_lie.OPS[name])
    trail_a = 2 if na == 9 else 1
    batch = tuple(a.shape[:-trail_a])
    if nb:
        batch = tuple(torch.broadcast_shapes(batch, tuple(b.shape[:-1])))
    return a.new_empty((*batch, *_lie._SHAPE.get(no, (no,))))


def _pose_loss_call(q, model, frame_ids, targets, weights):
    from . import _lib
    from .tree import device_tree
    m = _model(model)
    B = q.shape[0]
    dt = device_tree(m, q.device)
    ids = (_lib.c_int32 * len(frame_ids))(*frame_ids)
    loss = torch.empty(B, device=q.device, dtype=torch.float32)
    with torch.cuda.device(q.device):
        _lib.call("br_pose_loss", dt.ptr, q.data_ptr(), B, ids, len(frame_ids), targets.data_ptr(),
                  weights.data_ptr(), int(weights.dim() == 2), loss.data_ptr(), None, _lib.stream_ptr())
    return loss


@torch.library.custom_op("br_cuda::pose_loss", mutates_args=())
def pose_loss(q: torch.Tensor, model: int, frame_ids: Sequence[int], targets: torch.Tensor,
              weights: torch.Tensor) -> torch.Tensor:
    """``sum_f w_f |log(T_f^-1 oMf(q))|^2`` per configuration, ``(B,)``; q ``(B, nq)``,
    targets ``(B, F, 7)``, weights ``(F,)`` or ``(B, F)``.  Differentiable w.r.t. q (the
    backward is the adjoint kernel, FK recomputed)."""
    return _pose_loss_call(q.contiguous(), model, list(frame_ids), targets.contiguous(), weights.contiguous())


@pose_loss.register_fake
def _(q, model, frame_ids, targets, weights):
    return q.new_empty((q.shape[0],))


@torch.library.custom_op("br_cuda::pose_loss_backward", mutates_args=())
def pose_loss_backward(q: torch.Tensor, model: int, frame_ids: Sequence[int], targets: torch.Tensor,
                       weights: torch.Tensor, grad_loss: torch.Tensor) -> torch.Tensor:
    """Gradient of ``(grad_loss * pose_loss(q)).sum()`` w.r.t. raw q (free-flyer quaternion included)."""
    from . import _lib
    from .tree import device_tree
    m = _model(model)
    q = q.contiguous()
    grad_q = torch.empty_like(q)
    ids = (_lib.c_int32 * len(frame_ids))(*frame_ids)
    g = grad_loss.contiguous().float()
    with torch.cuda.device(q.device):
        _lib.call("br_pose_loss_backward", device_tree(m, q.device).ptr, q.data_ptr(), None, q.shape[0], ids,
                  len(frame_ids), targets.contiguous().data_ptr(), weights.contiguous().data_ptr(),
                  int(weights.dim() == 2), g.data_ptr(), grad_q.data_ptr(), _lib.stream_ptr())
    return grad_q


@pose_loss_backward.register_fake
def _(q, model, frame_ids, targets, weights, grad_loss):
    return torch.empty_like(q)


def _pose_loss_setup(ctx, inputs, output):
    q, model, frame_ids, targets, weights = inputs
    ctx.save_for_backward(q, targets, weights)
    ctx.model, ctx.frame_ids = model, list(frame_ids)


def _pose_loss_grad(ctx, grad_loss):
    q, targets, weights = ctx.saved_tensors
    return (torch.ops.br_cuda.pose_loss_backward(q, ctx.model, ctx.frame_ids, targets, weights, grad_loss),
            None, None, None, None)


pose_loss.register_autograd(_pose_loss_grad, setup_context=_pose_loss_setup)

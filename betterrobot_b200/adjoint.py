"""FK pose loss with a hand-written adjoint behind ``torch.autograd.Function``.

``pose_loss(model, q, frame_ids, targets, weights)`` returns, per configuration,
``sum_f w_f |log(T_f^-1 * oMf(q))|^2`` — the pose residual of
``src/better_robot/residuals/pose.py:58-66`` squared and summed over frames.
In the reference its gradient comes from torch autograd through every SE3 op
of the FK loop (``src/better_robot/kinematics/forward.py:79-81`` keeps that tape
on purpose); here ``backward`` is one CUDA kernel (``fk_adjoint.cu``).

Modes: ``"store"`` saves the world joint placements in the forward pass (read
back by the backward); ``"recompute"`` saves nothing and re-runs FK in the
backward; ``"auto"`` stores while ``batch * njoints * 28 B`` fits in the L2 cache.
"""

from __future__ import annotations

from typing import Sequence

import torch

from . import _lib
from .exceptions import ShapeError
from .kinematics import _validate_q
from .tree import device_tree


def choose_mode(model, batch: int, device) -> str:
    l2 = torch.cuda.get_device_properties(device).L2_cache_size
    return "store" if batch * model.njoints * 28 <= l2 else "recompute"


_IDS: dict = {}


def _ids(frame_ids: tuple):
    """The frame ids as a ctypes array, built once per id tuple."""
    arr = _IDS.get(frame_ids)
    if arr is None:
        if len(_IDS) >= 256:
            _IDS.clear()
        arr = _IDS[frame_ids] = (_lib.c_int32 * len(frame_ids))(*frame_ids)
    return arr


def _on_device(device, fn) -> None:
    """Run ``fn(stream)`` with ``device`` current (no context switch when it already is)."""
    if device.index == torch.cuda.current_device():
        fn(torch.cuda.current_stream().cuda_stream)
    else:
        with torch.cuda.device(device):
            fn(torch.cuda.current_stream().cuda_stream)


class _PoseLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, targets, weights, model, frame_ids, mode):
        B = q.shape[0]
        dt = device_tree(model, q.device)
        ids = _ids(frame_ids)
        loss = torch.empty(B, device=q.device, dtype=torch.float32)
        oMi = torch.empty(B, model.njoints, 7, device=q.device) if mode == "store" else None
        per_cfg = int(weights.dim() == 2)
        _on_device(q.device, lambda s: _lib.call(
            "br_pose_loss", dt.ptr, q.data_ptr(), B, ids, len(frame_ids), targets.data_ptr(), weights.data_ptr(),
            per_cfg, loss.data_ptr(), oMi.data_ptr() if oMi is not None else None, s))
        ctx.model, ctx.frame_ids, ctx.per_cfg = model, frame_ids, per_cfg
        if oMi is not None:
            ctx.save_for_backward(q, targets, weights, oMi)
        else:
            ctx.save_for_backward(q, targets, weights)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        saved = ctx.saved_tensors
        q, targets, weights = saved[:3]
        oMi = saved[3] if len(saved) > 3 else None
        g = grad_loss.contiguous().float()
        grad_q = torch.empty_like(q)
        dt = device_tree(ctx.model, q.device)
        ids = _ids(ctx.frame_ids)
        _on_device(q.device, lambda s: _lib.call(
            "br_pose_loss_backward", dt.ptr, q.data_ptr(), oMi.data_ptr() if oMi is not None else None,
            q.shape[0], ids, len(ctx.frame_ids), targets.data_ptr(), weights.data_ptr(), ctx.per_cfg,
            g.data_ptr(), grad_q.data_ptr(), s))
        return grad_q, None, None, None, None, None


def pose_loss(model, q: torch.Tensor, frame_ids: Sequence[int], targets: torch.Tensor, weights: torch.Tensor,
              mode: str = "auto", check_quaternion: bool = False) -> torch.Tensor:
    """Per-configuration pose loss ``(B,)``; differentiable w.r.t. ``q`` (B, nq) float32 CUDA.

    The backward kernel maps gradients to raw q for every joint kind of the tree table
    (fixed, revolute, unbounded revolute, prismatic, free-flyer, spherical, planar,
    translation).
    """
    _validate_q(model, q, check_quaternion)
    if q.dim() != 2:
        raise ShapeError("pose_loss takes q of shape (B, nq)")
    frame_ids = tuple(int(f) for f in frame_ids)
    B, F = q.shape[0], len(frame_ids)
    if targets.shape != (B, F, 7):
        raise ShapeError(f"targets must be ({B}, {F}, 7), got {tuple(targets.shape)}")
    if weights.shape not in ((F,), (B, F)):
        raise ShapeError(f"weights must be ({F},) or ({B}, {F}), got {tuple(weights.shape)}")
    if mode == "auto":
        mode = choose_mode(model, B, q.device)
    if mode not in ("store", "recompute"):
        raise ValueError(f"mode must be 'store', 'recompute' or 'auto', got {mode!r}")
    return _PoseLoss.apply(q.contiguous(), targets.contiguous().float(), weights.contiguous().float(), model,
                           frame_ids, mode)

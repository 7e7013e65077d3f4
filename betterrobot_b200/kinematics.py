"""Public kinematics surface, drop-in for ``better_robot.kinematics``.

Same names, arguments, shapes and exceptions as
``src/better_robot/kinematics/forward.py:35-219`` and
``src/better_robot/kinematics/jacobian.py:82-227``; the math runs in the fused
sm_100a kernels of ``libbr_b200.so``.  Inputs must be float32 CUDA tensors.
"""

from __future__ import annotations

from typing import Literal, Sequence

import torch

from . import _lib
from .data import Data, KinematicsLevel
from .exceptions import DeviceMismatchError, DtypeMismatchError, QuaternionNormError, ShapeError
from .tree import device_tree

ReferenceFrame = Literal["world", "local", "local_world_aligned"]
_REF = {"world": 0, "local_world_aligned": 1, "local": 2}
_QUAT_NORM_TOL = 0.1  # forward.py:32


def _ref_code(reference) -> int:
    key = getattr(reference, "value", reference)
    if key not in _REF:
        raise ValueError(f"Unsupported reference frame: {reference!r}")
    return _REF[key]


def _validate_q(model, q: torch.Tensor, check_quaternion: bool = True) -> None:
    """``_validate_q`` (``forward.py:35-70``) plus the CUDA/float32 requirements of this path."""
    if q.shape[-1] != model.nq:
        raise ShapeError(f"q has trailing size {q.shape[-1]}, expected model.nq={model.nq}")
    _lib.require_cuda(q)
    if q.dtype != torch.float32:
        raise DtypeMismatchError(f"q.dtype={q.dtype}; the sm_100a path computes in float32")
    if check_quaternion and model.njoints >= 2 and model.joint_models[1].kind == "free_flyer" and q.numel():
        norm = q[..., 3:7].norm(dim=-1)
        if bool(((norm - 1.0).abs() > _QUAT_NORM_TOL).any()):
            raise QuaternionNormError(
                f"free-flyer quaternion norm outside [{1 - _QUAT_NORM_TOL}, {1 + _QUAT_NORM_TOL}] "
                f"(observed range {(float(norm.min()), float(norm.max()))}). Normalise before passing.")


def _flat(q: torch.Tensor) -> torch.Tensor:
    return q.reshape(-1, q.shape[-1]).contiguous()


def forward_kinematics(model, q_or_data, *, compute_frames: bool = False, backend=None,
                       check_quaternion: bool = True) -> Data:
    """Joint placements (and frame placements if ``compute_frames``), ``forward.py:138-191``."""
    if isinstance(q_or_data, Data):
        data = q_or_data
        q = data.q
    else:
        q = q_or_data
        data = Data(q=q)
    _validate_q(model, q, check_quaternion)
    batch = tuple(q.shape[:-1])
    qf = _flat(q)
    B = qf.shape[0]
    dt = device_tree(model, q.device)
    oMi = torch.empty(B, model.njoints, 7, device=q.device, dtype=torch.float32)
    liMi = torch.empty_like(oMi)
    frames = None
    nf = 0
    ids = None
    if compute_frames:
        nf = int(model.nframes)
        frames = torch.empty(B, nf, 7, device=q.device, dtype=torch.float32)
    with torch.cuda.device(q.device):
        if compute_frames and nf > 64:
            _lib.call("br_forward_kinematics", dt.ptr, qf.data_ptr(), B, oMi.data_ptr(), liMi.data_ptr(),
                      None, 0, None, _lib.stream_ptr())
            for s in range(0, nf, 64):
                ids = (_lib.c_int32 * min(64, nf - s))(*range(s, min(nf, s + 64)))
                part = torch.empty(B, len(ids), 7, device=q.device)
                _lib.call("br_forward_kinematics", dt.ptr, qf.data_ptr(), B, None, None, ids, len(ids),
                          part.data_ptr(), _lib.stream_ptr())
                frames[:, s:s + len(ids)] = part
        else:
            if compute_frames:
                ids = (_lib.c_int32 * nf)(*range(nf))
            _lib.call("br_forward_kinematics", dt.ptr, qf.data_ptr(), B, oMi.data_ptr(), liMi.data_ptr(),
                      ids, nf, frames.data_ptr() if frames is not None else None, _lib.stream_ptr())
    object.__setattr__(data, "joint_pose_world", oMi.reshape(*batch, model.njoints, 7))
    object.__setattr__(data, "joint_pose_local", liMi.reshape(*batch, model.njoints, 7))
    object.__setattr__(data, "joint_jacobians", None)
    if frames is not None:
        object.__setattr__(data, "frame_pose_world", frames.reshape(*batch, nf, 7))
    object.__setattr__(data, "_kinematics_level", KinematicsLevel.PLACEMENTS)
    return data


def update_frame_placements(model, data: Data) -> Data:
    """``forward.py:194-219``: fill ``data.frame_pose_world`` for every frame."""
    data.require(KinematicsLevel.PLACEMENTS)
    fk = forward_kinematics(model, data.q, compute_frames=True, check_quaternion=False)
    object.__setattr__(data, "frame_pose_world", fk.frame_pose_world)
    return data


def _jac_from_poses(model, data: Data, targets: Sequence[int], reference) -> torch.Tensor:
    oMi = data.joint_pose_world
    batch = tuple(oMi.shape[:-2])
    of = oMi.reshape(-1, model.njoints, 7).contiguous()
    B = of.shape[0]
    dt = device_tree(model, oMi.device)
    out = torch.empty(B, len(targets), 6, model.nv, device=oMi.device, dtype=torch.float32)
    for s in range(0, len(targets), 64):
        chunk = list(targets[s:s + 64])
        ids = (_lib.c_int32 * len(chunk))(*chunk)
        dst = out if len(targets) <= 64 else torch.empty(B, len(chunk), 6, model.nv, device=oMi.device)
        with torch.cuda.device(oMi.device):
            _lib.call("br_frame_jacobians_from_poses", dt.ptr, of.data_ptr(), B, ids, len(chunk),
                      _ref_code(reference), dst.data_ptr(), _lib.stream_ptr())
        if dst is not out:
            out[:, s:s + len(chunk)] = dst
    return out.reshape(*batch, len(targets), 6, model.nv)


def get_frame_jacobian(model, data: Data, frame_id: int, *,
                       reference: ReferenceFrame = "local_world_aligned") -> torch.Tensor:
    """Frame Jacobian ``(B..., 6, nv)`` in ``world`` / ``local_world_aligned`` / ``local`` (``jacobian.py:129-227``)."""
    data.require(KinematicsLevel.PLACEMENTS)
    if not (0 <= int(frame_id) < model.nframes):
        raise IndexError(f"frame_id {frame_id} out of range for {model.nframes} frames")
    return _jac_from_poses(model, data, [int(frame_id)], reference)[..., 0, :, :]


def compute_joint_jacobians(model, data: Data, *, backend=None) -> Data:
    """World joint Jacobians ``(B..., njoints, 6, nv)`` into ``data.joint_jacobians`` (``jacobian.py:82-97``)."""
    data.require(KinematicsLevel.PLACEMENTS)
    J = _jac_from_poses(model, data, [-(j + 1) for j in range(model.njoints)], "world")
    object.__setattr__(data, "joint_jacobians", J)
    return data


def get_joint_jacobian(model, data: Data, joint_id: int, *, reference: ReferenceFrame = "world") -> torch.Tensor:
    """Joint Jacobian ``(B..., 6, nv)``; ``world`` or ``local`` = ``Ad(oMi^-1) J`` (``jacobian.py:100-126``)."""
    data.require(KinematicsLevel.PLACEMENTS)
    if reference == "world":
        if data.joint_jacobians is None:
            compute_joint_jacobians(model, data)
        return data.joint_jacobians[..., joint_id, :, :]
    if reference == "local":
        return _jac_from_poses(model, data, [-(int(joint_id) + 1)], "local")[..., 0, :, :]
    raise ValueError(f"Unsupported reference frame: {reference!r}")


def frame_jacobians(model, q: torch.Tensor, frame_ids: Sequence[int], *,
                    reference: ReferenceFrame = "local_world_aligned", return_poses: bool = True,
                    check_quaternion: bool = False):
    """Fused hot path: ``(oMf (B..., F, 7), J (B..., F, 6, nv))`` straight from ``q``.

    Equivalent to ``forward_kinematics(model, q, compute_frames=True)`` followed by
    ``get_frame_jacobian`` for each id in ``frame_ids`` (at most 64), in one kernel.
    """
    _validate_q(model, q, check_quaternion)
    frame_ids = [int(f) for f in frame_ids]
    if len(frame_ids) > 64:
        raise ShapeError("frame_jacobians takes at most 64 frames per call")
    batch = tuple(q.shape[:-1])
    qf = _flat(q)
    B = qf.shape[0]
    F = len(frame_ids)
    dt = device_tree(model, q.device)
    J = torch.empty(B, F, 6, model.nv, device=q.device, dtype=torch.float32)
    T = torch.empty(B, F, 7, device=q.device, dtype=torch.float32) if return_poses else None
    ids = (_lib.c_int32 * F)(*frame_ids)
    with torch.cuda.device(q.device):
        _lib.call("br_frame_jacobians", dt.ptr, qf.data_ptr(), B, ids, F, _ref_code(reference),
                  T.data_ptr() if T is not None else None, J.data_ptr(), _lib.stream_ptr())
    J = J.reshape(*batch, F, 6, model.nv)
    if T is None:
        return J
    return T.reshape(*batch, F, 7), J


def frame_jacobians_into(model, q: torch.Tensor, frame_ids, poses_out, jac_out, reference="local_world_aligned",
                         stream=None) -> None:
    """Allocation-free variant of ``frame_jacobians`` writing into caller buffers (for graphs / benchmarks)."""
    dt = device_tree(model, q.device)
    ids = (_lib.c_int32 * len(frame_ids))(*[int(f) for f in frame_ids])
    _lib.call("br_frame_jacobians", dt.ptr, q.data_ptr(), q.shape[0], ids, len(frame_ids), _ref_code(reference),
              poses_out.data_ptr() if poses_out is not None else None, jac_out.data_ptr(),
              stream if stream is not None else _lib.stream_ptr())

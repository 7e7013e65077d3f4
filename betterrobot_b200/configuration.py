"""Batched ``Model.integrate`` / ``Model.difference`` on the device.

Same semantics as ``src/better_robot/data_model/model.py:160-190`` (per joint:
``q + v`` / ``q1 - q0``; free-flyer ``normalize(q * exp(v))`` / ``log(q0^-1 * q1)``),
for float32 CUDA tensors with any leading batch shape.
"""

from __future__ import annotations

import torch

from . import _lib
from .exceptions import DtypeMismatchError, ShapeError
from .tree import device_tree

OP_INTEGRATE, OP_DIFFERENCE = 0, 1


def _check(t: torch.Tensor, n: int, name: str):
    if t.shape[-1] != n:
        raise ShapeError(f"{name} has trailing size {t.shape[-1]}, expected {n}")
    _lib.require_cuda(t)
    if t.dtype != torch.float32:
        raise DtypeMismatchError(f"{name}.dtype={t.dtype}; the sm_100a path computes in float32")


def _run(model, op, a, b, out_dim, out=None):
    batch = torch.broadcast_shapes(a.shape[:-1], b.shape[:-1])
    af = a.expand(*batch, a.shape[-1]).reshape(-1, a.shape[-1]).contiguous()
    bf = b.expand(*batch, b.shape[-1]).reshape(-1, b.shape[-1]).contiguous()
    if out is None:
        out = torch.empty(af.shape[0], out_dim, device=a.device, dtype=torch.float32)
    elif (out.shape[-1] != out_dim or out.numel() != af.shape[0] * out_dim or not out.is_contiguous()
          or out.dtype != torch.float32 or out.device != a.device):
        raise ShapeError(f"out must be a contiguous float32 ({af.shape[0]}, {out_dim}) tensor on {a.device}")
    dt = device_tree(model, a.device)
    with torch.cuda.device(a.device):
        _lib.call("br_configuration_op", dt.ptr, dt.active.data_ptr(), dt.n_active, op, af.data_ptr(), bf.data_ptr(),
                  af.shape[0], out.data_ptr(), _lib.stream_ptr())
    return out.reshape(*batch, out_dim)


def integrate(model, q: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """``q (+) v``: ``(B..., nq)``, ``(B..., nv)`` -> ``(B..., nq)``."""
    _check(q, model.nq, "q")
    _check(v, model.nv, "v")
    return _run(model, OP_INTEGRATE, q, v, model.nq)


def difference(model, q0: torch.Tensor, q1: torch.Tensor) -> torch.Tensor:
    """``q1 (-) q0``: two ``(B..., nq)`` -> ``(B..., nv)``."""
    _check(q0, model.nq, "q0")
    _check(q1, model.nq, "q1")
    return _run(model, OP_DIFFERENCE, q0, q1, model.nv)


def integrate_into(model, q: torch.Tensor, v: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
    """``integrate`` writing into a preallocated ``out`` (no allocation; graph-capturable)."""
    _check(q, model.nq, "q")
    _check(v, model.nv, "v")
    return _run(model, OP_INTEGRATE, q, v, model.nq, out)


def difference_into(model, q0: torch.Tensor, q1: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
    """``difference`` writing into a preallocated ``out``."""
    _check(q0, model.nq, "q0")
    _check(q1, model.nq, "q1")
    return _run(model, OP_DIFFERENCE, q0, q1, model.nv, out)

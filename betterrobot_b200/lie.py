"""Batched SE3 / SO3 primitives on the device (``br_lie_op``).

Same names, storage and broadcasting as ``better_robot.lie``'s torch backend
(``src/better_robot/lie/_torch_native_backend.py``): SE3 ``(..., 7)``
``[tx, ty, tz, qx, qy, qz, qw]``, SO3 ``(..., 4)`` scalar-last, tangents
``[v, w]`` linear first; adjoints and right Jacobians ``(..., 6, 6)``.  Inputs
are float32 CUDA tensors; leading dimensions broadcast.  No autograd: these are
the forward primitives of the kernels (gradients of FK losses come from
``betterrobot_b200.adjoint.pose_loss``).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from .exceptions import DtypeMismatchError, ShapeError

OPS = {
    "se3_compose": 0, "se3_inverse": 1, "se3_log": 2, "se3_exp": 3, "se3_act": 4, "se3_adjoint": 5,
    "se3_adjoint_inv": 6, "se3_normalize": 7, "so3_compose": 8, "so3_inverse": 9, "so3_log": 10, "so3_exp": 11,
    "so3_act": 12, "so3_to_matrix": 13, "so3_from_matrix": 14, "so3_normalize": 15, "right_jacobian_se3": 16,
    "right_jacobian_inv_se3": 17,
}
_SHAPE = {36: (6, 6), 9: (3, 3)}
_SIZES: dict[int, tuple[int, int, int]] = {}


def _sizes(op: int) -> tuple[int, int, int]:
    if op not in _SIZES:
        a, b, o = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _lib.call("br_lie_op_sizes", op, ctypes.byref(a), ctypes.byref(b), ctypes.byref(o))
        _SIZES[op] = (a.value, b.value, o.value)
    return _SIZES[op]


def _split(t: torch.Tensor, n: int, name: str) -> tuple[int, ...]:
    """Leading batch shape of ``t`` whose trailing shape must hold ``n`` floats per element."""
    _lib.require_cuda(t)
    if t.dtype != torch.float32:
        raise DtypeMismatchError(f"{name}.dtype={t.dtype}; the sm_100a path computes in float32")
    trail = _SHAPE.get(n, (n,))
    if t.dim() < len(trail) or tuple(t.shape[-len(trail):]) != trail:
        raise ShapeError(f"{name} has shape {tuple(t.shape)}, expected trailing {trail}")
    return tuple(t.shape[:-len(trail)])


def _flat(t: torch.Tensor, batch: tuple[int, ...], own: tuple[int, ...], n: int) -> tuple[torch.Tensor, int]:
    """(contiguous (N, n) tensor, count), count 1 when ``t`` holds one element that broadcasts."""
    numel = 1
    for s in own:
        numel *= s
    if numel == 1:
        return t.reshape(1, n).contiguous(), 1
    e = t.reshape(*own, n).expand(*batch, n)
    return e.reshape(-1, n).contiguous(), e.shape[:-1].numel()


def apply(name: str, a: torch.Tensor, b: torch.Tensor | None = None) -> torch.Tensor:
    """``out = op(a, b)`` elementwise over the broadcast batch."""
    op = OPS[name]
    na_f, nb_f, no_f = _sizes(op)
    ba = _split(a, na_f, "a")
    if nb_f:
        if b is None:
            raise TypeError(f"{name} takes two operands")
        bb = _split(b, nb_f, "b")
        if b.device != a.device:
            raise ShapeError("operands are on different devices")
        batch = tuple(torch.broadcast_shapes(ba, bb))
    else:
        bb, batch = (), ba
    n = 1
    for s in batch:
        n *= s
    af, na = _flat(a, batch, ba, na_f)
    bf, nb = _flat(b, batch, bb, nb_f) if nb_f else (None, 0)
    out = torch.empty(n, no_f, device=a.device, dtype=torch.float32)
    with torch.cuda.device(a.device):
        _lib.call("br_lie_op", op, af.data_ptr(), na, bf.data_ptr() if bf is not None else None, nb,
                  out.data_ptr(), n, _lib.stream_ptr())
    return out.reshape(*batch, *_SHAPE.get(no_f, (no_f,)))


def se3_compose(a, b): return apply("se3_compose", a, b)            # noqa: E704
def se3_inverse(t): return apply("se3_inverse", t)                 # noqa: E704
def se3_log(t): return apply("se3_log", t)                         # noqa: E704
def se3_exp(xi): return apply("se3_exp", xi)                       # noqa: E704
def se3_act(t, p): return apply("se3_act", t, p)                   # noqa: E704
def se3_adjoint(t): return apply("se3_adjoint", t)                 # noqa: E704
def se3_adjoint_inv(t): return apply("se3_adjoint_inv", t)         # noqa: E704
def se3_normalize(t): return apply("se3_normalize", t)             # noqa: E704
def so3_compose(a, b): return apply("so3_compose", a, b)           # noqa: E704
def so3_inverse(q): return apply("so3_inverse", q)                 # noqa: E704
def so3_log(q): return apply("so3_log", q)                         # noqa: E704
def so3_exp(w): return apply("so3_exp", w)                         # noqa: E704
def so3_act(q, p): return apply("so3_act", q, p)                   # noqa: E704
def so3_to_matrix(q): return apply("so3_to_matrix", q)             # noqa: E704
def so3_from_matrix(R): return apply("so3_from_matrix", R)         # noqa: E704
def so3_normalize(q): return apply("so3_normalize", q)             # noqa: E704
def right_jacobian_se3(xi): return apply("right_jacobian_se3", xi)  # noqa: E704
def right_jacobian_inv_se3(xi): return apply("right_jacobian_inv_se3", xi)  # noqa: E704


class B200LieOps:
    """``LieOps`` (``src/better_robot/backends/protocol.py:27-51``) on the device kernels."""

    se3_compose = staticmethod(se3_compose)
    se3_inverse = staticmethod(se3_inverse)
    se3_log = staticmethod(se3_log)
    se3_exp = staticmethod(se3_exp)
    se3_act = staticmethod(se3_act)
    se3_adjoint = staticmethod(se3_adjoint)
    se3_adjoint_inv = staticmethod(se3_adjoint_inv)
    se3_normalize = staticmethod(se3_normalize)
    so3_compose = staticmethod(so3_compose)
    so3_inverse = staticmethod(so3_inverse)
    so3_log = staticmethod(so3_log)
    so3_exp = staticmethod(so3_exp)
    so3_act = staticmethod(so3_act)
    so3_to_matrix = staticmethod(so3_to_matrix)
    so3_from_matrix = staticmethod(so3_from_matrix)
    so3_normalize = staticmethod(so3_normalize)

"""A BetterRobot ``Backend`` whose kinematics and Lie ops run on the sm_100a kernels.

BetterRobot routes forward kinematics and joint Jacobians through
``backend.kinematics`` (``src/better_robot/backends/protocol.py:55-69``, called from
``src/better_robot/kinematics/forward.py:181-183`` and
``src/better_robot/kinematics/jacobian.py:95-96``) and every SE3 / SO3 op through
``backend.lie`` (``src/better_robot/lie/se3.py:28-29``).  Any object with
``name``, ``lie``, ``kinematics`` and ``dynamics`` (``protocol.py:113-119``) can be
passed as ``backend=`` to those public functions, so::

    from betterrobot_b200.backend import BACKEND
    data = better_robot.forward_kinematics(model, q_cuda_f32, backend=BACKEND)

runs BetterRobot's own FK entry point on ``br_forward_kinematics``.  Inputs must be
float32 CUDA tensors; anything else raises (there is no CPU path).  Dynamics are
outside this package: ``dynamics`` is whatever the caller supplies (for example the
torch-native ``DynamicsOps``), else a stub that raises.
"""

from __future__ import annotations

import functools

import torch

from . import kinematics as _kin
from .exceptions import BackendNotAvailableError, ShapeError
from .lie import B200LieOps


class B200KinematicsOps:
    """``KinematicsOps`` (``protocol.py:55-69``) on ``libbr_b200.so``."""

    def forward_kinematics(self, model, q: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """``(joint_pose_world, joint_pose_local)``, each ``(B..., njoints, 7)``.

        The caller (``forward.py:181``) has already validated ``q``; like the torch
        backend, this trusts it.  There is no autograd through this op: a ``q`` that
        requires grad raises (differentiate FK losses with ``adjoint.pose_loss``).
        """
        if q.requires_grad:
            raise BackendNotAvailableError(
                "the b200 kinematics backend does not record autograd; use betterrobot_b200.adjoint.pose_loss "
                "for gradients of pose losses, or the torch_native backend")
        data = _kin.forward_kinematics(model, q, check_quaternion=False)
        return data.joint_pose_world, data.joint_pose_local

    def compute_joint_jacobians(self, model, data) -> torch.Tensor:
        """World joint Jacobians ``(B..., njoints, 6, nv)`` from ``data.joint_pose_world``."""
        if getattr(data, "joint_pose_world", None) is None:
            raise ShapeError("data.joint_pose_world is not populated; run forward_kinematics first")
        return _kin._jac_from_poses(model, data, [-(j + 1) for j in range(model.njoints)], "world")


class _NoDynamics:
    """Placeholder ``DynamicsOps``: rigid-body dynamics are not part of this package."""

    def _raise(self, *_a, **_k):
        raise BackendNotAvailableError(
            "rigid-body dynamics are not implemented by the b200 backend; pass dynamics= to B200Backend")

    rnea = aba = crba = center_of_mass = _raise


class B200Backend:
    """``Backend`` bundle (``protocol.py:113-119``) named ``"b200"``."""

    name: str = "b200"

    def __init__(self, *, lie=None, dynamics=None) -> None:
        self.lie = lie if lie is not None else B200LieOps()
        self.kinematics = B200KinematicsOps()
        self.dynamics = dynamics if dynamics is not None else _NoDynamics()


BACKEND = B200Backend()


def graph_capture(fn=None, *, warmup: int = 2):
    """Decorator: run ``fn`` as a replayed CUDA graph, one graph per argument signature.

    The reference's ``better_robot.backends.graph_capture`` (``backends/__init__.py:110-127``)
    is the seam for this and is a no-op on its torch backend.  Here the first call with a
    new signature (shapes, dtypes, devices of the tensor arguments plus the values of the
    others) runs ``fn`` ``warmup`` times on a side stream, then captures one call into a
    ``torch.cuda.CUDAGraph`` that reads static copies of the tensor arguments.  Later
    calls copy the arguments into those buffers and replay the graph.

    ``fn`` must be capturable: no host synchronisation (``.item()``, ``bool(tensor)``),
    no allocation that changes with the data.  The kernels of this package launch on the
    current stream and can be captured.  The returned tensors are the graph's static
    outputs and are overwritten by the next replay; clone to keep them.
    """
    if fn is None:
        return functools.partial(graph_capture, warmup=warmup)
    graphs: dict = {}

    def key_of(args, kwargs):
        def k(x):
            if isinstance(x, torch.Tensor):
                return ("T", tuple(x.shape), x.dtype, str(x.device))
            return ("V", x)
        return tuple(k(a) for a in args) + tuple((n, k(v)) for n, v in sorted(kwargs.items()))

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        key = key_of(args, kwargs)
        entry = graphs.get(key)
        if entry is None:
            sargs = [a.clone() if isinstance(a, torch.Tensor) else a for a in args]
            skw = {n: (v.clone() if isinstance(v, torch.Tensor) else v) for n, v in kwargs.items()}
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                for _ in range(warmup):
                    fn(*sargs, **skw)
            torch.cuda.current_stream().wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                out = fn(*sargs, **skw)
            entry = (g, sargs, skw, out)
            graphs[key] = entry
        g, sargs, skw, out = entry
        for dst, src in zip(sargs, args):
            if isinstance(dst, torch.Tensor):
                dst.copy_(src)
        for n, v in kwargs.items():
            if isinstance(skw[n], torch.Tensor):
                skw[n].copy_(v)
        g.replay()
        return out

    wrapper.graphs = graphs
    return wrapper

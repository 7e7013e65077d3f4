"""Batched kinematic trajectory optimisation on the sm_100a nested-dissection solver.

Counterpart of ``solve_trajopt`` with the knot parameterisation
(``src/better_robot/tasks/trajopt.py:84-230``) for the cost stack
goal pose at the last knot + start pose at the first knot + acceleration
smoothness + per-knot joint limits + reference trajectory
(``TimeIndexedResidual(PoseResidual)``, ``AccelerationResidual``,
``TimeIndexedResidual(JointPositionLimit)``, ``ReferenceTrajectoryResidual``),
solved by Gauss-Newton (or LM) for many trajectories in one launch.  Returns
also the adjoint gradient of the final cost w.r.t. the goal pose.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib
from .exceptions import UnsupportedJointError, ShapeError
from .tree import device_tree


@dataclass
class TrajOptConfig:
    dt: float = 0.05
    w_goal: float = 1.0
    w_start: float = 1.0
    w_accel: float = 1e-2
    w_limit: float = 0.1
    w_ref: float = 1e-3
    optimizer: str = "gn"           # "gn" | "lm"
    max_iter: int = 30
    tol: float = 1e-6
    gn_eps: float = 1e-8
    lam0: float = 1e-3
    factor: float = 10.0


@dataclass
class BatchTrajResult:
    q: torch.Tensor            # (N, T, nq)
    iters: torch.Tensor        # (N,)
    converged: torch.Tensor    # (N,)
    status: torch.Tensor
    cost: torch.Tensor         # (N,) final 0.5 |r|^2
    goal_grad: torch.Tensor | None  # (N, 6) d cost / d eps, goal -> goal * exp(eps)


def settings_from(cfg: TrajOptConfig) -> _lib.TrajSettings:
    if cfg.optimizer not in ("gn", "lm"):
        raise NotImplementedError(f"optimizer {cfg.optimizer!r}: the sm_100a trajopt runs 'gn' and 'lm'")
    s = _lib.TrajSettings()
    s.dt, s.w_goal, s.w_start, s.w_accel, s.w_limit, s.w_ref = cfg.dt, cfg.w_goal, cfg.w_start, cfg.w_accel, \
        cfg.w_limit, cfg.w_ref
    s.tol, s.gn_eps, s.lam0, s.factor, s.lam_min, s.lam_max = cfg.tol, cfg.gn_eps, cfg.lam0, cfg.factor, 1e-10, 1e8
    s.max_iter = int(cfg.max_iter)
    s.optimizer = 0 if cfg.optimizer == "lm" else 1
    return s


def solve_trajopt_batched(model, frame_id: int, goal: torch.Tensor, initial_q_traj: torch.Tensor, *,
                          start: torch.Tensor | None = None, q_ref: torch.Tensor | None = None,
                          cfg: TrajOptConfig | None = None, want_goal_grad: bool = True) -> BatchTrajResult:
    """``initial_q_traj (N, T, nq)``, ``goal (N, 7)`` (and ``start (N, 7)``) float32 CUDA tensors."""
    bad = [jm.kind for jm in model.joint_models
           if not (jm.kind in ("universe", "fixed", "translation", "free_flyer", "spherical", "planar")
                   or jm.kind.startswith("prismatic") or jm.kind.startswith("revolute"))]
    if bad:
        raise UnsupportedJointError(f"trajopt: no knot difference / retraction for joint kinds {sorted(set(bad))}")
    cfg = cfg or TrajOptConfig()
    if initial_q_traj.dim() != 3 or initial_q_traj.shape[-1] != model.nq:
        raise ShapeError(f"initial_q_traj must be (N, T, {model.nq}), got {tuple(initial_q_traj.shape)}")
    _lib.require_cuda(initial_q_traj)
    N, T, nq = initial_q_traj.shape
    if goal.shape != (N, 7) or (start is not None and start.shape != (N, 7)):
        raise ShapeError("goal / start must be (N, 7)")
    x0 = initial_q_traj.contiguous().float()
    dev = x0.device
    x = torch.empty_like(x0)
    iters = torch.empty(N, dtype=torch.int32, device=dev)
    status = torch.empty(N, dtype=torch.int32, device=dev)
    cost = torch.empty(N, device=dev)
    gg = torch.empty(N, 6, device=dev) if want_goal_grad else None
    goal_c = goal.contiguous().float()
    start_c = start.contiguous().float() if start is not None else None
    ref_c = q_ref.contiguous().float() if q_ref is not None else None
    dt = device_tree(model, dev)
    with torch.cuda.device(dev):
        _lib.call("br_trajopt_solve", dt.ptr, int(frame_id), N, T, x0.data_ptr(),
                  ref_c.data_ptr() if ref_c is not None else None, goal_c.data_ptr(),
                  start_c.data_ptr() if start_c is not None else None, settings_from(cfg), x.data_ptr(),
                  iters.data_ptr(), status.data_ptr(), cost.data_ptr(), gg.data_ptr() if gg is not None else None,
                  _lib.stream_ptr())
    return BatchTrajResult(q=x, iters=iters, converged=(status & 0xFF) == 0, status=status, cost=cost, goal_grad=gg)

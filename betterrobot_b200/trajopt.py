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


@dataclass
class Trajectory:
    """Knot trajectory of a ``solve_trajopt`` result (the fields of ``tasks/trajectory.py``'s
    ``Trajectory`` that ``solve_trajopt`` fills: times ``(1, T)``, configurations ``(1, T, nq)``)."""

    t: torch.Tensor
    q: torch.Tensor
    model_id: int = -1


@dataclass
class TrajOptResult:
    """Return type of ``solve_trajopt`` (``tasks/trajopt.py:71-84``); ``cost`` is the final
    ``0.5 |r|^2`` (the reference returns the stacked residual instead)."""

    trajectory: Trajectory
    cost: float
    iters: int
    converged: bool
    model: object
    goal_grad: torch.Tensor | None = None


def _stack_to_config(model, cost_stack, horizon: int, optimizer, max_iter: int):
    """Read a BetterRobot ``CostStack`` (``costs/stack.py:25-60``: ``items`` name -> ``CostItem``
    with ``residual``, ``weight``, ``active``) into the kernel's fixed stack.  Recognised items:
    ``TimeIndexedResidual(PoseResidual, t_idx=T-1)`` (goal) and ``t_idx=0`` (start) on one frame,
    ``AccelerationResidual``, ``TimeIndexedResidual(JointPositionLimit, t_idx=t)`` for every knot t
    with one weight, ``ReferenceTrajectoryResidual``; effective weights are item weight x the
    residual's own weight.  Anything else raises ``NotImplementedError``."""
    items = [it for it in getattr(cost_stack, "items", {}).values() if getattr(it, "active", True)]
    if not items:
        raise ShapeError("solve_trajopt: the cost stack has no active item")
    cfg = TrajOptConfig(w_goal=0.0, w_start=0.0, w_accel=0.0, w_limit=0.0, w_ref=0.0, max_iter=int(max_iter))
    frame_id, goal, start, q_ref = None, None, None, None
    limit_knots, limit_w = set(), None
    for it in items:
        r, w = it.residual, float(it.weight)
        kind = type(r).__name__
        if kind == "TimeIndexedResidual" and type(r.inner).__name__ == "PoseResidual":
            pr = r.inner
            if float(pr.pos_weight) != float(pr.ori_weight):
                raise NotImplementedError("solve_trajopt: pose terms need pos_weight == ori_weight")
            if frame_id is not None and int(pr.frame_id) != frame_id:
                raise NotImplementedError("solve_trajopt: goal and start poses must be of one frame")
            frame_id = int(pr.frame_id)
            t_idx = int(r.t_idx) % horizon
            if t_idx == horizon - 1:
                goal, cfg.w_goal = pr.target, w * float(pr.pos_weight)
            elif t_idx == 0:
                start, cfg.w_start = pr.target, w * float(pr.pos_weight)
            else:
                raise NotImplementedError("solve_trajopt: pose terms only at the first and last knot")
        elif kind == "TimeIndexedResidual" and type(r.inner).__name__ == "JointPositionLimit":
            wi = w * float(r.inner.weight)
            if limit_w is not None and wi != limit_w:
                raise NotImplementedError("solve_trajopt: per-knot limit terms need one weight")
            limit_w = wi
            limit_knots.add(int(r.t_idx) % horizon)
        elif kind == "AccelerationResidual":
            cfg.w_accel, cfg.dt = w * float(r.weight), float(r.dt)
        elif kind == "ReferenceTrajectoryResidual":
            cfg.w_ref, q_ref = w * float(r.weight), r.q_ref
        else:
            raise NotImplementedError(f"solve_trajopt: residual {kind} is not on the sm_100a trajectory path")
    if limit_knots and limit_knots != set(range(horizon)):
        raise NotImplementedError("solve_trajopt: joint limit terms must cover every knot")
    cfg.w_limit = limit_w or 0.0
    if goal is None:
        raise NotImplementedError("solve_trajopt: the stack needs a pose term at the last knot")
    opt = type(optimizer).__name__
    if opt == "GaussNewton":
        cfg.optimizer, cfg.tol, cfg.gn_eps = "gn", float(optimizer.tol), float(getattr(optimizer, "eps", 1e-8))
    elif opt == "LevenbergMarquardt":
        cfg.optimizer, cfg.tol = "lm", float(optimizer.tol)
        cfg.lam0, cfg.factor = float(optimizer.lam0), float(optimizer.factor)
    else:
        raise NotImplementedError(f"solve_trajopt: optimizer {opt}; the sm_100a path runs GaussNewton and "
                                  "LevenbergMarquardt")
    return cfg, frame_id, goal, start, q_ref


def solve_trajopt(model, *, horizon: int, dt: float, initial_q_traj: torch.Tensor, cost_stack, optimizer,
                  max_iter: int = 50, jacobian_strategy=None, lower=None, upper=None,
                  parameterization=None) -> TrajOptResult:
    """Drop-in for ``better_robot.solve_trajopt`` (``tasks/trajopt.py:84-230``) with the knot
    parameterisation, for the stack the kernel solves (see ``_stack_to_config``): one
    trajectory ``initial_q_traj (T, nq)`` through ``br_trajopt_solve``.  For many trajectories
    at once use ``solve_trajopt_batched``."""
    if initial_q_traj.dim() != 2:
        raise ValueError(f"initial_q_traj must be (T, nq); got {tuple(initial_q_traj.shape)}")
    T, nq = initial_q_traj.shape
    if T != horizon:
        raise ValueError(f"horizon={horizon} inconsistent with initial_q_traj.shape[0]={T}")
    if nq != model.nq:
        raise ValueError(f"initial_q_traj.shape[1]={nq} != model.nq={model.nq}")
    if parameterization is not None and type(parameterization).__name__ != "KnotTrajectory":
        raise NotImplementedError("solve_trajopt: the sm_100a path optimises knots (KnotTrajectory)")
    if lower is not None or upper is not None:
        raise NotImplementedError("solve_trajopt: box clamps are not on the sm_100a path; use limit terms")
    cfg, fid, goal, start, q_ref = _stack_to_config(model, cost_stack, T, optimizer, max_iter)
    dev = initial_q_traj.device if initial_q_traj.is_cuda else torch.device("cuda")
    X0 = initial_q_traj.detach().to(dev, torch.float32)[None]
    as_pose = lambda p: torch.as_tensor(p).detach().to(dev, torch.float32).reshape(1, 7)  # noqa: E731
    ref = torch.as_tensor(q_ref).detach().to(dev, torch.float32).reshape(1, T, nq) if q_ref is not None else None
    out = solve_trajopt_batched(model, fid, as_pose(goal), X0, start=as_pose(start) if start is not None else None,
                                q_ref=ref, cfg=cfg)
    t_axis = torch.linspace(0.0, (T - 1) * dt, T, device=dev)
    return TrajOptResult(trajectory=Trajectory(t=t_axis[None], q=out.q, model_id=getattr(model, "id", -1)),
                         cost=float(out.cost[0]), iters=int(out.iters[0]), converged=bool(out.converged[0]),
                         model=model, goal_grad=out.goal_grad)

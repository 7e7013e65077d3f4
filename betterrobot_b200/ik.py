"""Batched LM / Gauss-Newton IK on the sm_100a persistent kernel.

Drop-in for ``better_robot.tasks.ik`` (``src/better_robot/tasks/ik.py:37-266``):
``solve_ik(model, targets, initial_q=..., cost_cfg=..., optimizer_cfg=...)`` builds
the same cost stack — one ``PoseResidual`` per target, ``JointPositionLimit``
(item weight ``limit_weight``), ``RestResidual`` (item weight ``rest_weight``) —
and runs the same Levenberg-Marquardt loop with ``Adaptive`` damping.  Unlike
the reference it also solves whole batches, including uneven mixes of robots,
in one launch (``solve_ik_batched``, ``PackedIK``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Literal, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import BrTree, IKBatch, IKResultBuf, IKSettings, c_int32
from .exceptions import ShapeError
from .tree import device_tree

OPT_LM, OPT_GN = 0, 1
MAX_CLASSES, MAX_TARGETS = 8, 8
SCRATCH_BYTES = 16


@dataclass
class IKCostConfig:
    """Weights of the built-in IK stack (``tasks/ik.py:37-48``)."""

    pos_weight: float = 1.0
    ori_weight: float = 1.0
    pose_weight: float = 1.0
    limit_weight: float = 0.1
    rest_weight: float = 0.01
    collision_margin: float = 0.02
    collision_weight: float = 1.0
    q_rest: torch.Tensor | None = None


@dataclass
class OptimizerConfig:
    """Optimizer selection (``tasks/ik.py:51-69``).

    ``lam0``/``factor`` are the ``Adaptive`` damping parameters; their defaults are
    what ``solve_ik`` effectively uses (``Adaptive()`` = 1e-4 / 2, ``tasks/ik.py:250``).
    ``lam_min``/``lam_max`` are ``Adaptive``'s clamps (``strategies/adaptive.py:19-25``).
    """

    optimizer: Literal["lm", "gn", "adam", "lbfgs", "lm_then_lbfgs"] = "lm"
    max_iter: int = 100
    jacobian_strategy: object = None
    linear_solver: Literal["cholesky", "lstsq", "cg"] = "cholesky"
    kernel: Literal["l2", "huber", "cauchy", "tukey"] = "l2"
    damping: Literal["constant", "adaptive", "trust_region"] = "adaptive"
    tol: float = 1e-6
    refine_disabled_items: tuple = ()
    lam0: float = 1e-4
    factor: float = 2.0
    lam_min: float = 1e-10
    lam_max: float = 1e8
    gn_eps: float = 1e-8
    kernel_param: float | None = None  # None: the kernel class's default (Huber 1.0, Cauchy 1.0, Tukey 4.685)
    # arithmetic of the Jacobian, J^T J, J^T r and the factorization ("f32": fastest; "f64": the
    # float64 reference's iterates); the iterate, FK, residual and cost are float64 in both
    precision: Literal["f32", "f64"] = "f32"


PRECISIONS = {"f32": 0, "f64": 1}  # BR_PREC_*


# OptimizerConfig.kernel -> BR_KERNEL_*, and the default parameter of each kernel class
# (src/better_robot/optim/kernels/huber.py, cauchy.py, tukey.py)
KERNELS = {"l2": 0, "huber": 1, "cauchy": 2, "tukey": 3}
TARGET_KINDS = {"pose": 0, "position": 1, "orientation": 2}   # BR_TARGET_*
KERNEL_DEFAULTS = {"huber": 1.0, "cauchy": 1.0, "tukey": 4.685}


@dataclass
class IKResult:
    """Return type of ``solve_ik`` (``tasks/ik.py:72-99``)."""

    q: torch.Tensor
    residual: torch.Tensor
    iters: int
    converged: bool
    model: object

    def fk(self):
        from .kinematics import forward_kinematics
        return forward_kinematics(self.model, self.q, compute_frames=True)

    def frame_pose(self, name: str) -> torch.Tensor:
        return self.fk().frame_pose_world[..., self.model.frame_id(name), :]

    def q_only(self) -> torch.Tensor:
        return self.q


@dataclass
class BatchIKResult:
    """Batched result: ``q (P, nq)`` (or a list for uneven mixes), per-problem iterations/verdicts."""

    q: object
    iters: torch.Tensor
    converged: torch.Tensor
    status: torch.Tensor
    cost: torch.Tensor
    residual: object = None


def settings_from(cost_cfg: IKCostConfig, opt: OptimizerConfig) -> IKSettings:
    if opt.optimizer not in ("lm", "gn"):
        raise NotImplementedError(f"optimizer {opt.optimizer!r}: the sm_100a path runs 'lm' and 'gn'")
    if opt.linear_solver != "cholesky":
        raise NotImplementedError("the sm_100a path solves the normal equations by Cholesky")
    if opt.damping not in ("adaptive", "constant"):
        raise NotImplementedError(f"damping {opt.damping!r} is not on the sm_100a path")
    s = IKSettings()
    s.lam0 = opt.lam0
    s.factor = 1.0 if opt.damping == "constant" else opt.factor   # Constant: lambda never changes
    s.tol = opt.tol
    s.lam_min, s.lam_max, s.gn_eps = opt.lam_min, opt.lam_max, opt.gn_eps
    s.pos_weight = cost_cfg.pos_weight * cost_cfg.pose_weight       # tasks/ik.py:193-194
    s.ori_weight = cost_cfg.ori_weight * cost_cfg.pose_weight
    s.limit_weight = cost_cfg.limit_weight
    s.rest_weight = cost_cfg.rest_weight
    s.max_iter = int(opt.max_iter)
    s.optimizer = OPT_LM if opt.optimizer == "lm" else OPT_GN
    if opt.kernel not in KERNELS:
        raise ValueError(f"Unknown kernel {opt.kernel!r}; expected one of {sorted(KERNELS)}")
    s.kernel = KERNELS[opt.kernel]
    s.kernel_param = KERNEL_DEFAULTS.get(opt.kernel, 0.0) if opt.kernel_param is None else float(opt.kernel_param)
    if opt.precision not in PRECISIONS:
        raise ValueError(f"Unknown precision {opt.precision!r}; expected 'f32' or 'f64'")
    s.precision = PRECISIONS[opt.precision]
    return s


def team_floats(model, max_targets: int, device) -> int:
    dt = device_tree(model, device)
    return int(_lib.load().br_lm_team_floats(dt.ptr, max_targets))


def default_team_size(model) -> int:
    """Lanes per problem: the kernel is built for 32-lane teams only."""
    return 32


class PackedIK:
    """An uneven batch of IK problems packed for one persistent launch.

    ``problems`` are grouped by robot (class).  For class ``c``: ``models[c]``,
    ``frame_ids[c]`` (P_c, K_c) int, ``targets[c]`` (P_c, K_c, 7) float32,
    ``q0[c]`` (P_c, nq_c) float32 and ``n_targets[c]`` (P_c,) (<= K_c).
    Device buffers are allocated once; ``set_inputs`` refreshes targets / q0 in place
    and ``solve`` launches (graph-capturable: no allocation, no host sync).
    """

    def __init__(self, models: Sequence, frame_ids: Sequence, n_targets: Sequence, q_rest: Sequence | None = None,
                 team_sizes: Sequence[int] | None = None, device="cuda", warps_per_cta: int = 4,
                 with_residual: bool = False, target_kinds: Sequence | None = None):
        if not 1 <= len(models) <= MAX_CLASSES:
            raise ShapeError(f"1..{MAX_CLASSES} robot classes per launch, got {len(models)}")
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.models = list(models)
        self.C = len(models)
        self.counts = [int(np.asarray(n).shape[0]) for n in n_targets]
        self.P = sum(self.counts)
        self.K = max(int(np.asarray(f).shape[1]) for f in frame_ids)
        if self.K > MAX_TARGETS:
            raise ShapeError(f"at most {MAX_TARGETS} targets per problem")
        self.team = [int(t) for t in (team_sizes or [default_team_size(m) for m in models])]
        for m, t in zip(models, self.team):
            if t != 32:
                raise ShapeError(f"team size {t}: the kernel runs one problem per 32-lane warp")
        self.trees = [device_tree(m, self.device) for m in models]
        self.warps_per_cta = warps_per_cta
        # per-problem layout: classes contiguous, in class order
        self.class_start = np.cumsum([0] + self.counts)[:-1]
        nq = np.concatenate([np.full(n, m.nq, np.int64) for n, m in zip(self.counts, models)])
        # P + 1 offsets (the last one is the total), so a class with no problems indexes in range
        self.q_offset_np = np.concatenate([[0], np.cumsum(nq)]).astype(np.int64)
        self.q_total = int(nq.sum())
        nt_all = np.concatenate([np.asarray(n, np.int32) for n in n_targets])
        if (nt_all < 1).any() or (nt_all > self.K).any():
            raise ShapeError("each problem needs 1..K targets")
        fr = np.zeros((self.P, self.K), np.int32)
        for c in range(self.C):
            f = np.asarray(frame_ids[c], np.int32)
            if f.size and (f.min() < 0 or f.max() >= models[c].nframes):
                raise ShapeError(f"class {c}: frame id out of range")
            s0 = self.class_start[c]
            fr[s0:s0 + self.counts[c], :f.shape[1]] = f
        kinds = np.zeros((self.P, self.K), np.int32)
        if target_kinds is not None:
            for c in range(self.C):
                if target_kinds[c] is None:
                    continue
                k = np.asarray([TARGET_KINDS[x] if isinstance(x, str) else int(x)
                                for x in np.asarray(target_kinds[c]).reshape(-1)], np.int32)
                k = k.reshape(np.asarray(target_kinds[c]).shape)
                if ((k < 0) | (k > 2)).any():
                    raise ShapeError("target kinds are 'pose', 'position' or 'orientation'")
                s0 = self.class_start[c]
                kinds[s0:s0 + self.counts[c], :k.shape[-1]] = np.broadcast_to(k, (self.counts[c], k.shape[-1]))
        rows = np.where(kinds == 0, 6, 3) * (np.arange(self.K)[None, :] < nt_all[:, None])
        dims = []
        for c, m in enumerate(models):
            s0 = self.class_start[c]
            dims.append(rows[s0:s0 + self.counts[c]].sum(-1) + 2 * m.nq + m.nv)
        rdim = np.concatenate(dims)
        self.r_offset_np = np.concatenate([[0], np.cumsum(rdim)]).astype(np.int64)
        self.r_dim = rdim
        # work items: heaviest classes first, and inside a class the problems with the fewest
        # targets first (they run the most iterations: a less constrained problem's rest term
        # settles slowly), so the longest solves start early and the launch's tail is short
        cost = [m.nv ** 2 * (1 + self.K) for m in models]
        order, items = [], []
        slot = 0
        for c in sorted(range(self.C), key=lambda k: -cost[k]):
            per = 32 // self.team[c]
            s0 = int(self.class_start[c])
            idx = s0 + np.argsort(nt_all[s0:s0 + self.counts[c]], kind="stable")
            order.append(idx)
            for s in range(0, self.counts[c], per):
                items.append((slot + s, min(per, self.counts[c] - s), c))
            slot += self.counts[c]
        dev = self.device
        self.order = torch.from_numpy(np.concatenate(order).astype(np.int32)).to(dev)
        self.items = torch.tensor(items, dtype=torch.int32, device=dev).reshape(-1)
        self.n_items = len(items)
        self.n_targets_t = torch.from_numpy(nt_all).to(dev)
        self.frames_t = torch.from_numpy(fr).to(dev)
        self.q_offset = torch.from_numpy(self.q_offset_np).to(dev)
        self.r_offset = torch.from_numpy(self.r_offset_np).to(dev)
        self.kinds = torch.from_numpy(kinds).to(dev) if kinds.any() else None
        self.targets = torch.zeros(self.P, self.K, 7, device=dev)
        self.targets[..., 6] = 1.0
        self.x0 = torch.zeros(self.q_total, device=dev)
        self.q_rest = torch.zeros(self.q_total, device=dev)
        for c, m in enumerate(models):
            qr = (m.q_neutral if q_rest is None or q_rest[c] is None else q_rest[c])
            qr = torch.as_tensor(qr, dtype=torch.float32).reshape(-1, m.nq)
            s0 = int(self.q_offset_np[self.class_start[c]])
            self.q_rest[s0:s0 + self.counts[c] * m.nq] = qr.to(dev).expand(self.counts[c], m.nq).reshape(-1)
        self.x = torch.empty(self.q_total, device=dev)
        self.iters = torch.empty(self.P, dtype=torch.int32, device=dev)
        self.status = torch.empty(self.P, dtype=torch.int32, device=dev)
        self.cost = torch.empty(self.P, device=dev)
        # fixed layout per problem: target rows, 2 nq limit rows, nv rest rows (zero when unused)
        self.residual = torch.zeros(int(rdim.sum()), device=dev) if with_residual else None
        self.scratch = torch.zeros(SCRATCH_BYTES // 4, dtype=torch.int32, device=dev)
        # ctypes structs (kept alive on the object)
        self._trees = (BrTree * self.C)(*[t.struct for t in self.trees])
        self._teams = (c_int32 * self.C)(*self.team)
        b = IKBatch()
        b.n_problems, b.max_targets, b.n_classes, b.n_items = self.P, self.K, self.C, self.n_items
        b.trees = ctypes.cast(self._trees, ctypes.POINTER(BrTree))
        b.team_size = ctypes.cast(self._teams, ctypes.POINTER(c_int32))
        b.items, b.order = self.items.data_ptr(), self.order.data_ptr()
        b.n_targets, b.frames = self.n_targets_t.data_ptr(), self.frames_t.data_ptr()
        b.targets, b.q_offset = self.targets.data_ptr(), self.q_offset.data_ptr()
        b.x0, b.q_rest = self.x0.data_ptr(), self.q_rest.data_ptr()
        b.r_offset = self.r_offset.data_ptr()
        b.target_kind = self.kinds.data_ptr() if self.kinds is not None else None
        self._batch = b
        r = IKResultBuf()
        r.x, r.iters, r.status, r.cost = self.x.data_ptr(), self.iters.data_ptr(), self.status.data_ptr(), \
            self.cost.data_ptr()
        r.residual = self.residual.data_ptr() if self.residual is not None else None
        self._result = r

    def set_inputs(self, targets: Sequence, q0: Sequence) -> None:
        """Copy per-class targets (P_c, K_c, 7) and start configurations (P_c, nq_c) into the device buffers."""
        for c, m in enumerate(self.models):
            s0, n = int(self.class_start[c]), self.counts[c]
            t = torch.as_tensor(targets[c], dtype=torch.float32)
            self.targets[s0:s0 + n, :t.shape[1]].copy_(t, non_blocking=True)
            o = int(self.q_offset_np[s0])
            self.x0[o:o + n * m.nq].copy_(torch.as_tensor(q0[c], dtype=torch.float32).reshape(-1), non_blocking=True)

    def solve(self, settings: IKSettings, stream: int | None = None) -> None:
        _lib.call("br_lm_solve", ctypes.byref(self._batch), ctypes.byref(settings), ctypes.byref(self._result),
                  self.warps_per_cta, self.scratch.data_ptr(), SCRATCH_BYTES,
                  stream if stream is not None else _lib.stream_ptr(self.device))

    def capture(self, settings: IKSettings) -> "torch.cuda.CUDAGraph":
        """Capture one solve (scratch zeroing + the persistent launch) in a CUDA graph.

        Replaying the graph re-solves from the current contents of the input buffers
        (``set_inputs`` copies new targets / start configurations into them in place).
        """
        self._graph_settings = settings  # the struct must outlive the capture call
        with torch.cuda.device(self.device):
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                self.solve(settings)           # warm-up outside capture (module load, smem attribute)
            torch.cuda.current_stream().wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.solve(settings)
        self.graph = g
        return g

    def q_of(self, c: int) -> torch.Tensor:
        s0, n, nq = int(self.class_start[c]), self.counts[c], self.models[c].nq
        o = int(self.q_offset_np[s0])
        return self.x[o:o + n * nq].view(n, nq)

    def class_slice(self, c: int) -> slice:
        s0 = int(self.class_start[c])
        return slice(s0, s0 + self.counts[c])


def solve_ik_batched(model, frame_ids, targets: torch.Tensor, initial_q: torch.Tensor, *,
                     cost_cfg: IKCostConfig | None = None, optimizer_cfg: OptimizerConfig | None = None,
                     n_targets=None, with_residual: bool = False, team_size: int | None = None,
                     warps_per_cta: int = 4, target_kinds=None) -> BatchIKResult:
    """Solve ``P`` independent problems of one robot: ``targets (P, K, 7)`` for ``frame_ids``
    (K ids shared by all problems, or ``(P, K)``), ``initial_q (P, nq)``.

    ``target_kinds`` (K names, or a ``(P, K)`` array): "pose" (``PoseResidual``, the
    default), "position" (``PositionResidual``, weight ``pos_weight * pose_weight``) or
    "orientation" (``OrientationResidual``, weight ``ori_weight * pose_weight``),
    ``src/better_robot/residuals/pose.py:58-195``.  With ``with_residual`` the stacked
    residual has 6 rows per pose target and 3 per position / orientation target.
    """
    cost_cfg = cost_cfg or IKCostConfig()
    optimizer_cfg = optimizer_cfg or OptimizerConfig()
    if initial_q.dim() != 2 or initial_q.shape[-1] != model.nq:
        raise ShapeError(f"initial_q must be (P, {model.nq}), got {tuple(initial_q.shape)}")
    _lib.require_cuda(initial_q)
    P = initial_q.shape[0]
    fr = np.asarray(frame_ids, np.int32)
    if fr.ndim == 1:
        fr = np.broadcast_to(fr, (P, fr.shape[0]))
    K = fr.shape[1]
    if targets.shape != (P, K, 7):
        raise ShapeError(f"targets must be ({P}, {K}, 7), got {tuple(targets.shape)}")
    nt = np.full(P, K, np.int32) if n_targets is None else np.asarray(n_targets, np.int32)
    qr = [cost_cfg.q_rest] if cost_cfg.q_rest is not None else None
    pk = PackedIK([model], [fr], [nt], q_rest=qr, team_sizes=[team_size or default_team_size(model)],
                  device=initial_q.device, warps_per_cta=warps_per_cta, with_residual=with_residual,
                  target_kinds=None if target_kinds is None else [target_kinds])
    pk.set_inputs([targets], [initial_q])
    with torch.cuda.device(initial_q.device):
        pk.solve(settings_from(cost_cfg, optimizer_cfg))
    res = None
    if with_residual:
        # the reference's CostStack has a limit / rest block only when its weight is > 0
        # (tasks/ik.py:200-205): drop the unused blocks of the fixed device layout
        def stack_rows(r: torch.Tensor) -> torch.Tensor:
            nt_rows = r.shape[-1] - 2 * model.nq - model.nv
            parts = [r[..., :nt_rows]]
            if cost_cfg.limit_weight > 0.0:
                parts.append(r[..., nt_rows:nt_rows + 2 * model.nq])
            if cost_cfg.rest_weight > 0.0:
                parts.append(r[..., nt_rows + 2 * model.nq:])
            return torch.cat(parts, -1) if len(parts) > 1 else parts[0]
        if P == 0:
            res = pk.residual.view(0, 0)
        else:
            res = (stack_rows(pk.residual.view(P, -1)) if (pk.r_dim == pk.r_dim[0]).all()
                   else [stack_rows(r) for r in torch.split(pk.residual, [int(d) for d in pk.r_dim])])
    return BatchIKResult(q=pk.q_of(0), iters=pk.iters, converged=(pk.status & 0xFF) == 0, status=pk.status,
                         cost=pk.cost, residual=res)


def solve_ik(model, targets: dict, *, initial_q: torch.Tensor | None = None, cost_cfg: IKCostConfig | None = None,
             optimizer_cfg: OptimizerConfig | None = None, robot_collision=None, device=None) -> IKResult:
    """Whole-body IK for one configuration (``tasks/ik.py:150-266``); ``targets``: frame name -> (7,) pose."""
    cost_cfg = cost_cfg or IKCostConfig()
    optimizer_cfg = optimizer_cfg or OptimizerConfig()
    if initial_q is not None:
        x0 = initial_q.detach().float()
    else:
        x0 = model.q_neutral.clone().float()
    dev = x0.device if x0.is_cuda else torch.device(device or "cuda")
    x0 = x0.to(dev).reshape(1, -1)
    names = list(targets)
    if not names:
        raise ShapeError("solve_ik needs at least one target")
    fids = [model.frame_id(n) for n in names]
    T = torch.stack([torch.as_tensor(targets[n], dtype=torch.float32).reshape(7) for n in names]).to(dev)
    out = solve_ik_batched(model, fids, T[None], x0, cost_cfg=cost_cfg, optimizer_cfg=optimizer_cfg,
                           with_residual=True)
    return IKResult(q=out.q[0], residual=out.residual[0], iters=int(out.iters[0]), converged=bool(out.converged[0]),
                    model=model)

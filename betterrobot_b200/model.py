"""Kinematic-tree description with the reference ``Model``'s field names.

The hot path accepts either this ``Model`` or BetterRobot's own
``better_robot.data_model.model.Model`` (``src/better_robot/data_model/model.py:22-205``):
both expose the same attributes that the device packer reads — ``parents``,
``topo_order``, ``joint_models[j].kind/.nq/.nv/.axis``, ``nqs/nvs/idx_qs/idx_vs``,
``joint_placements (njoints, 7)``, ``lower/upper_pos_limit (nq,)``, ``frames`` and
``q_neutral``.  This module exists so that the GPU path runs where BetterRobot
itself is not installed; it builds the same joint numbering as the reference's
``build_model`` (universe = joint 0, root = joint 1, then a depth-first preorder,
``src/better_robot/io/build_model.py:158-182``) and the same frame list
(``body_<name>`` for every body, then the operational frames, ``build_model.py:451-466``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence

import torch

# Joint kinds understood by the device tree table.  Names are the reference's
# ``JointModel.kind`` strings (``src/better_robot/data_model/joint_models/*.py``).
REVOLUTE_KINDS = ("revolute_rx", "revolute_ry", "revolute_rz", "revolute_unaligned")
PRISMATIC_KINDS = ("prismatic_px", "prismatic_py", "prismatic_pz", "prismatic_unaligned")
FIXED_KINDS = ("universe", "fixed")
FREE_FLYER_KIND = "free_flyer"
# multi-slot kinds: (nq, nv) and neutral configuration (joint_models/*.py)
MULTI_KINDS = {"spherical": (4, 3, (0.0, 0.0, 0.0, 1.0)), "planar": (4, 3, (0.0, 0.0, 1.0, 0.0)),
               "revolute_unbounded": (2, 1, (1.0, 0.0)), "translation": (3, 3, (0.0, 0.0, 0.0))}

_AXES = {
    "revolute_rx": (1.0, 0.0, 0.0), "revolute_ry": (0.0, 1.0, 0.0), "revolute_rz": (0.0, 0.0, 1.0),
    "prismatic_px": (1.0, 0.0, 0.0), "prismatic_py": (0.0, 1.0, 0.0), "prismatic_pz": (0.0, 0.0, 1.0),
}

IDENTITY_SE3 = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)


@dataclass(frozen=True)
class JointModel:
    """Per-joint kind record (``kind``, ``nq``, ``nv``, ``axis``) as on the reference's joint models."""

    kind: str
    nq: int
    nv: int
    axis: torch.Tensor | None = None

    def neutral(self) -> torch.Tensor:
        if self.kind == FREE_FLYER_KIND:
            return torch.tensor(IDENTITY_SE3)
        if self.kind in MULTI_KINDS:
            return torch.tensor(MULTI_KINDS[self.kind][2])
        return torch.zeros(self.nq)


def joint_model(kind: str, axis: Sequence[float] | None = None) -> JointModel:
    """Return the ``JointModel`` for a reference kind string (axis used for ``*_unaligned``)."""
    if kind in FIXED_KINDS:
        return JointModel(kind, 0, 0, None)
    if kind == FREE_FLYER_KIND:
        return JointModel(kind, 7, 6, None)
    if kind in MULTI_KINDS:
        nq, nv, _ = MULTI_KINDS[kind]
        ax = None
        if kind == "revolute_unbounded":  # axis defaults to z (revolute.py:195-198)
            ax = torch.tensor([float(a) for a in (axis if axis is not None else (0.0, 0.0, 1.0))])
        return JointModel(kind, nq, nv, ax)
    if kind in REVOLUTE_KINDS or kind in PRISMATIC_KINDS:
        if kind.endswith("unaligned"):
            if axis is None:
                raise ValueError(f"{kind} needs an axis")
            return JointModel(kind, 1, 1, torch.tensor([float(a) for a in axis]))
        return JointModel(kind, 1, 1, None)
    from .exceptions import UnsupportedJointError
    raise UnsupportedJointError(f"joint kind {kind!r} is not supported by the sm_100a path")


def kind_for_axis(family: str, axis: Sequence[float]) -> str:
    """Map an axis to the reference's aligned kind (``build_model._kind_to_joint_model``, ``io/build_model.py:106-134``)."""
    a = tuple(float(x) for x in axis)
    names = {(1.0, 0.0, 0.0): "x", (0.0, 1.0, 0.0): "y", (0.0, 0.0, 1.0): "z"}
    for ref, s in names.items():
        if max(abs(a[i] - ref[i]) for i in range(3)) < 1e-6:
            return f"revolute_r{s}" if family == "revolute" else f"prismatic_p{s}"
    return f"{family}_unaligned"


def joint_axis(jm) -> tuple[float, float, float]:
    """Local joint axis of a revolute/prismatic joint model (reference or local)."""
    kind = jm.kind
    if kind in _AXES:
        return _AXES[kind]
    ax = getattr(jm, "axis", None)
    if ax is None and kind == "revolute_unbounded":
        return (0.0, 0.0, 1.0)
    if ax is None:
        return (0.0, 0.0, 0.0)
    ax = ax.detach().cpu().double().reshape(-1).tolist()
    return (ax[0], ax[1], ax[2])


@dataclass(frozen=True)
class Frame:
    """Named placement rigidly attached to ``parent_joint`` (``src/better_robot/data_model/frame.py:21-28``)."""

    name: str
    parent_joint: int
    joint_placement: torch.Tensor
    frame_type: str = "op"


def _topology(parents: tuple[int, ...]):
    n = len(parents)
    children: list[list[int]] = [[] for _ in range(n)]
    for j, p in enumerate(parents):
        if p >= 0:
            children[p].append(j)
    order: list[int] = []
    stack = [0]
    while stack:
        j = stack.pop()
        order.append(j)
        stack.extend(reversed(sorted(children[j])))
    supports: list[tuple[int, ...]] = [()] * n
    for j in order:
        p = parents[j]
        supports[j] = (j,) if p < 0 else supports[p] + (j,)
    return tuple(tuple(sorted(c)) for c in children), tuple(order), tuple(supports)


@dataclass(frozen=True)
class Model:
    """Frozen kinematic tree; field names follow ``src/better_robot/data_model/model.py:22-85``."""

    njoints: int
    nframes: int
    nq: int
    nv: int
    name: str
    joint_names: tuple[str, ...]
    frame_names: tuple[str, ...]
    joint_name_to_id: dict
    frame_name_to_id: dict
    parents: tuple[int, ...]
    children: tuple[tuple[int, ...], ...]
    supports: tuple[tuple[int, ...], ...]
    topo_order: tuple[int, ...]
    joint_models: tuple[JointModel, ...]
    nqs: tuple[int, ...]
    nvs: tuple[int, ...]
    idx_qs: tuple[int, ...]
    idx_vs: tuple[int, ...]
    joint_placements: torch.Tensor
    lower_pos_limit: torch.Tensor
    upper_pos_limit: torch.Tensor
    frames: tuple[Frame, ...]
    q_neutral: torch.Tensor = field(default_factory=lambda: torch.zeros(0))

    def frame_id(self, name: str) -> int:
        return self.frame_name_to_id[name]

    def joint_id(self, name: str) -> int:
        return self.joint_name_to_id[name]

    def get_support(self, joint_id: int) -> tuple[int, ...]:
        return self.supports[joint_id]

    def to(self, device=None, dtype=None) -> "Model":
        import dataclasses
        t = lambda x: x.to(device=device, dtype=dtype)  # noqa: E731
        return dataclasses.replace(
            self, joint_placements=t(self.joint_placements), lower_pos_limit=t(self.lower_pos_limit),
            upper_pos_limit=t(self.upper_pos_limit), q_neutral=t(self.q_neutral))


def build_model(name: str, joints: Sequence[dict], frames: Sequence[dict] = (),
                dtype: torch.dtype = torch.float32) -> Model:
    """Build a ``Model`` from joint records already in depth-first preorder.

    ``joints[i]`` describes model joint ``i + 1`` (joint 0 is the universe) with keys
    ``name``, ``kind`` (reference kind string), ``parent`` (model joint index),
    ``origin`` (7,), optional ``axis``, ``lower``, ``upper``, ``body``.
    ``frames`` are operational frames ``{name, parent, placement}`` appended after
    the per-body ``body_<name>`` frames, as ``build_model`` does.
    """
    inf = float("inf")
    names = ["universe"]
    bodies = ["universe"]
    parents = [-1]
    jms: list[JointModel] = [JointModel("universe", 0, 0, None)]
    placements = [torch.tensor(IDENTITY_SE3, dtype=torch.float64)]
    lower: list[float] = []
    upper: list[float] = []
    for i, rec in enumerate(joints):
        j = i + 1
        p = int(rec["parent"])
        if not (0 <= p < j):
            raise ValueError(f"joint {rec['name']!r}: parent {p} must precede it (preorder)")
        jm = joint_model(rec["kind"], rec.get("axis"))
        names.append(rec["name"])
        bodies.append(rec.get("body", f"{rec['name']}_link"))
        parents.append(p)
        jms.append(jm)
        placements.append(torch.as_tensor(rec.get("origin", IDENTITY_SE3), dtype=torch.float64))
        if jm.kind == FREE_FLYER_KIND:
            lower.extend([-inf] * 7)
            upper.extend([inf] * 7)
        elif jm.kind in MULTI_KINDS:  # the limits build_model gives these kinds (io/build_model.py:382-408)
            lo, hi = {"spherical": ([-1.0] * 4, [1.0] * 4), "planar": ([-inf, -inf, -1.0, -1.0], [inf, inf, 1.0, 1.0]),
                      "revolute_unbounded": ([-inf] * 2, [inf] * 2), "translation": ([-inf] * 3, [inf] * 3)}[jm.kind]
            lower.extend(lo)
            upper.extend(hi)
        elif jm.nq == 1:
            lo = rec.get("lower")
            hi = rec.get("upper")
            lower.append(-inf if lo is None else float(lo))
            upper.append(inf if hi is None else float(hi))
    nqs = tuple(jm.nq for jm in jms)
    nvs = tuple(jm.nv for jm in jms)
    idx_qs, idx_vs, oq, ov = [], [], 0, 0
    for a, b in zip(nqs, nvs):
        idx_qs.append(oq)
        idx_vs.append(ov)
        oq += a
        ov += b
    parents_t = tuple(parents)
    children, order, supports = _topology(parents_t)
    frame_list = [Frame(f"body_{b}", j, torch.tensor(IDENTITY_SE3, dtype=dtype), "body")
                  for j, b in enumerate(bodies)]
    for fr in frames:
        frame_list.append(Frame(fr["name"], int(fr["parent"]),
                                torch.as_tensor(fr.get("placement", IDENTITY_SE3), dtype=torch.float64).to(dtype),
                                fr.get("frame_type", "op")))
    q_neutral = torch.cat([jm.neutral() for jm in jms if jm.nq > 0]) if oq else torch.zeros(0)
    return Model(
        njoints=len(jms), nframes=len(frame_list), nq=oq, nv=ov, name=name,
        joint_names=tuple(names), frame_names=tuple(f.name for f in frame_list),
        joint_name_to_id={n: i for i, n in enumerate(names)},
        frame_name_to_id={f.name: i for i, f in enumerate(frame_list)},
        parents=parents_t, children=children, supports=supports, topo_order=order,
        joint_models=tuple(jms), nqs=nqs, nvs=nvs, idx_qs=tuple(idx_qs), idx_vs=tuple(idx_vs),
        joint_placements=torch.stack(placements).to(dtype),
        lower_pos_limit=torch.tensor(lower, dtype=dtype), upper_pos_limit=torch.tensor(upper, dtype=dtype),
        frames=tuple(frame_list), q_neutral=q_neutral.to(dtype),
    )

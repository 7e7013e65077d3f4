"""Pack a ``Model`` into the device tree table (``br_tree_t``).

Reads only the attributes shared by this package's ``Model`` and BetterRobot's
(``src/better_robot/data_model/model.py:22-85``), so either can be passed.  The
table is built once per (model, device) and cached, matching the frozen-Model
contract of the reference (``model.py:21-29``).
"""

from __future__ import annotations

import ctypes
import math
import weakref

import numpy as np
import torch

from ._lib import BrTree
from .exceptions import ModelInconsistencyError, UnsupportedJointError
from .model import FIXED_KINDS, FREE_FLYER_KIND, PRISMATIC_KINDS, REVOLUTE_KINDS, joint_axis

JOINT_FIXED, JOINT_REVOLUTE, JOINT_PRISMATIC, JOINT_FREE_FLYER = 0, 1, 2, 3
JOINT_SPHERICAL, JOINT_PLANAR, JOINT_REVOLUTE_UNBOUNDED, JOINT_TRANSLATION = 4, 5, 6, 7
# tangent columns of the multi-slot kinds in the joint frame: (col_kind 0 = rotation about,
# 1 = translation along, axis) — the motion subspaces of joint_models/{spherical,planar,translation}.py
_MULTI_COLUMNS = {
    "spherical": (JOINT_SPHERICAL, [(0, 0), (0, 1), (0, 2)]),
    "planar": (JOINT_PLANAR, [(1, 0), (1, 1), (0, 2)]),
    "translation": (JOINT_TRANSLATION, [(1, 0), (1, 1), (1, 2)]),
}
MAX_JOINTS, MAX_NV, MAX_NQ = 64, 64, 128


def _np(x) -> np.ndarray:
    if hasattr(x, "detach"):
        return x.detach().cpu().double().numpy()
    return np.asarray(x, dtype=np.float64)


class TreeArrays:
    """Host (numpy) arrays of one tree table."""

    def __init__(self, model):
        nj, nq, nv = int(model.njoints), int(model.nq), int(model.nv)
        if nj > MAX_JOINTS or nv > MAX_NV or nq > MAX_NQ:
            raise UnsupportedJointError(
                f"model {getattr(model, 'name', '?')!r} has njoints={nj}, nv={nv}, nq={nq}; "
                f"the device tree table holds at most {MAX_JOINTS} joints, nv {MAX_NV}, nq {MAX_NQ}")
        parents = tuple(int(p) for p in model.parents)
        if parents[0] != -1 or any(not (0 <= parents[j] < j) for j in range(1, nj)):
            raise ModelInconsistencyError("parents must satisfy parents[0] == -1 and parents[j] < j")
        self.nj, self.nq, self.nv, self.nf = nj, nq, nv, int(model.nframes)
        self.parent = np.array(parents, dtype=np.int32)
        self.jtype = np.zeros(nj, np.int32)
        self.idx_q = np.array(model.idx_qs, dtype=np.int32)
        self.idx_v = np.array(model.idx_vs, dtype=np.int32)
        self.axis = np.zeros((nj, 4), np.float32)
        self.placement = np.zeros((nj, 8), np.float32)
        P = _np(model.joint_placements)
        self.placement[:, :3] = P[:, :3]
        self.placement[:, 4:8] = P[:, 3:7]
        self.col_joint = np.zeros(nv, np.int32)
        self.col_kind = np.zeros(nv, np.int32)
        self.col_axis = np.zeros((nv, 4), np.float32)
        for j, jm in enumerate(model.joint_models):
            kind = jm.kind
            iv = int(model.idx_vs[j])
            if kind in FIXED_KINDS:
                self.jtype[j] = JOINT_FIXED
            elif kind in REVOLUTE_KINDS or kind in PRISMATIC_KINDS:
                rev = kind in REVOLUTE_KINDS
                self.jtype[j] = JOINT_REVOLUTE if rev else JOINT_PRISMATIC
                a = joint_axis(jm)
                self.axis[j, :3] = a
                self.col_joint[iv] = j
                self.col_kind[iv] = 0 if rev else 1
                self.col_axis[iv, :3] = a
            elif kind == "revolute_unbounded":
                self.jtype[j] = JOINT_REVOLUTE_UNBOUNDED
                a = joint_axis(jm)
                self.axis[j, :3] = a
                self.col_joint[iv] = j
                self.col_kind[iv] = 0
                self.col_axis[iv, :3] = a
            elif kind in _MULTI_COLUMNS:
                self.jtype[j], cols = _MULTI_COLUMNS[kind]
                for k, (ck, ax) in enumerate(cols):
                    self.col_joint[iv + k] = j
                    self.col_kind[iv + k] = ck
                    self.col_axis[iv + k, ax] = 1.0
            elif kind == FREE_FLYER_KIND:
                self.jtype[j] = JOINT_FREE_FLYER
                for k in range(6):
                    self.col_joint[iv + k] = j
                    self.col_kind[iv + k] = 1 if k < 3 else 0
                    self.col_axis[iv + k, k % 3] = 1.0
            else:
                raise UnsupportedJointError(f"joint {j} has kind {kind!r}, not encoded by the sm_100a tree table")
            if (int(jm.nq), int(jm.nv)) != (int(model.nqs[j]), int(model.nvs[j])):
                raise ModelInconsistencyError(f"joint {j}: nq/nv disagree with the model tables")
        depth = np.zeros(nj, np.int64)
        support = np.zeros(nj, np.uint64)
        for j in range(nj):
            p = parents[j]
            depth[j] = 0 if p < 0 else depth[p] + 1
            support[j] = (np.uint64(0) if p < 0 else support[p]) | np.uint64(1 << j)
        self.support = support
        self.rounds = int(math.ceil(math.log2(int(depth.max()) + 1))) if nj > 1 else 0
        self.frame_parent = np.array([int(f.parent_joint) for f in model.frames], dtype=np.int32)
        if self.nf and (self.frame_parent.min() < 0 or self.frame_parent.max() >= nj):
            raise ModelInconsistencyError("frame parent joint out of range")
        if (self.idx_q + np.array(model.nqs) > nq).any() or (self.idx_v + np.array(model.nvs) > nv).any():
            raise ModelInconsistencyError("joint q/v slices exceed nq/nv")
        # slices are laid out cumulatively in joint order, as data_model/model.py builds idx_qs / idx_vs
        if (np.cumsum([0, *model.nqs[:-1]]) != self.idx_q).any() or (np.cumsum([0, *model.nvs[:-1]]) != self.idx_v).any():
            raise ModelInconsistencyError("idx_qs / idx_vs must be cumulative in joint order")
        self.frame_placement = np.zeros((self.nf, 8), np.float32)
        for i, f in enumerate(model.frames):
            fp = _np(f.joint_placement)
            self.frame_placement[i, :3] = fp[:3]
            self.frame_placement[i, 4:8] = fp[3:7]
        # DOF tree (a joint's DOFs chained, the first under the last DOF of the nearest
        # ancestor joint with DOFs): J^T J entries per DOF = depth + 1
        lastd = np.full(nj, -1, np.int64)
        ddep = np.zeros(nv, np.int64)
        self.dof_parent = np.full(nv, -1, np.int32)
        for j in range(nj):
            p = parents[j]
            prev = lastd[p] if p >= 0 else -1
            nvj = int(model.nvs[j])
            for k in range(nvj):
                c = int(self.idx_v[j]) + k
                pc = prev if k == 0 else c - 1
                self.dof_parent[c] = pc
                ddep[c] = 0 if pc < 0 else ddep[pc] + 1
            lastd[j] = int(self.idx_v[j]) + nvj - 1 if nvj else prev
        self.dof_entries = int((ddep + 1).sum())
        self.dof_depth = int(ddep.max()) + 1 if nv else 1
        self.lower = _np(model.lower_pos_limit).astype(np.float32)
        self.upper = _np(model.upper_pos_limit).astype(np.float32)

    def sections(self):
        return [("parent", self.parent), ("jtype", self.jtype), ("idx_q", self.idx_q), ("idx_v", self.idx_v),
                ("axis", self.axis), ("placement", self.placement), ("support", self.support),
                ("frame_parent", self.frame_parent), ("frame_placement", self.frame_placement),
                ("col_joint", self.col_joint), ("col_kind", self.col_kind), ("col_axis", self.col_axis),
                ("lower", self.lower), ("upper", self.upper)]

    def dof_schedule(self) -> np.ndarray:
        """The LM's level schedule over the DOF tree (``br_dof_schedule``, host code of the library)."""
        from . import _lib
        lib = _lib.load()
        dp = np.ascontiguousarray(self.dof_parent)
        n = lib.br_dof_schedule(dp.ctypes.data, self.nv, None, 0)
        if n < 0:
            raise ModelInconsistencyError(f"br_dof_schedule failed ({n})")
        out = np.zeros(max(int(n), 4), np.uint32)
        n2 = lib.br_dof_schedule(dp.ctypes.data, self.nv, out.ctypes.data, out.size)
        if n2 != n:
            raise ModelInconsistencyError(f"br_dof_schedule failed ({n2})")
        return out

    def blob(self, extra=()) -> tuple[np.ndarray, dict]:
        """One byte buffer with 16-byte aligned sections, and their offsets."""
        offs, parts, o = {}, [], 0
        for name, arr in [*self.sections(), *extra]:
            b = np.ascontiguousarray(arr).tobytes()
            offs[name] = o
            pad = (-len(b)) % 16
            parts.append(b + b"\0" * pad)
            o += len(b) + pad
        buf = np.frombuffer(b"".join(parts) or b"\0" * 16, dtype=np.uint8).copy()
        return buf, offs


class DeviceTree:
    """Tree table resident on one CUDA device plus its ``br_tree_t`` struct."""

    def __init__(self, model, device: torch.device):
        self._model = _weak(model)
        self.arrays = TreeArrays(model)
        sched = self.arrays.dof_schedule() if self.arrays.nv else None
        buf, offs = self.arrays.blob([("dof_sched", sched)] if sched is not None else [])
        self.buffer = torch.from_numpy(buf).to(device)
        base = self.buffer.data_ptr()
        a = self.arrays
        st = BrTree()
        st.njoints, st.nq, st.nv, st.nframes, st.rounds = a.nj, a.nq, a.nv, a.nf, a.rounds
        st.kinds = int(np.bitwise_or.reduce(np.left_shift(1, a.jtype.astype(np.int64))))
        st.dof_entries, st.dof_depth = a.dof_entries, a.dof_depth
        for name, _ in a.sections():
            setattr(st, name, base + offs[name])
        st.dof_sched = base + offs["dof_sched"] if sched is not None else None
        self.struct = st
        self.ptr = ctypes.pointer(st)
        self.device = device
        act = [j for j in range(a.nj) if int(model.nqs[j]) > 0]
        self.active = torch.tensor(act or [0], dtype=torch.int32, device=device)
        self.n_active = len(act)


    @property
    def model(self):
        """The model this table was built from (None once it has been garbage collected)."""
        return self._model()


def _weak(model):
    """A weak reference to ``model``, or a strong one for objects that cannot be weakly referenced."""
    try:
        return weakref.ref(model)
    except TypeError:
        return lambda: model


# (id(model), device) -> DeviceTree.  Entries refer to their model weakly and are dropped
# when it is collected, so the cache keeps no model (nor its device table) alive.
_CACHE: dict[tuple[int, str], DeviceTree] = {}


def _drop(key) -> None:
    _CACHE.pop(key, None)


def device_tree(model, device) -> DeviceTree:
    device = torch.device(device)
    if device.type == "cuda" and device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    key = (id(model), str(device))
    dt = _CACHE.get(key)
    if dt is None or dt.model is not model:
        dt = DeviceTree(model, device)
        _CACHE[key] = dt
        try:
            weakref.finalize(model, _drop, key)
        except TypeError:
            pass
    return dt

"""``Data`` workspace with the reference's field names (``src/better_robot/data_model/data.py``).

Only the kinematics fields of the hot path are kept.  Reassigning ``q``
invalidates the cached placements and Jacobians, as ``Data.__setattr__`` does in
the reference; reading a field before it is computed raises ``StaleCacheError``
through ``require``.
"""

from __future__ import annotations

import enum
from dataclasses import dataclass
from typing import Optional

import torch

from .exceptions import StaleCacheError


class KinematicsLevel(enum.IntEnum):
    NONE = 0
    PLACEMENTS = 1


@dataclass
class Data:
    q: torch.Tensor
    joint_pose_world: Optional[torch.Tensor] = None   # (B..., njoints, 7)  oMi
    joint_pose_local: Optional[torch.Tensor] = None   # (B..., njoints, 7)  liMi
    frame_pose_world: Optional[torch.Tensor] = None   # (B..., nframes, 7)  oMf
    joint_jacobians: Optional[torch.Tensor] = None    # (B..., njoints, 6, nv)
    _kinematics_level: KinematicsLevel = KinematicsLevel.NONE

    def __setattr__(self, name, value):
        object.__setattr__(self, name, value)
        if name == "q" and hasattr(self, "_kinematics_level"):
            for f in ("joint_pose_world", "joint_pose_local", "frame_pose_world", "joint_jacobians"):
                object.__setattr__(self, f, None)
            object.__setattr__(self, "_kinematics_level", KinematicsLevel.NONE)

    def require(self, level: KinematicsLevel) -> None:
        if int(self._kinematics_level) < int(level):
            raise StaleCacheError(
                f"Data holds kinematics level {self._kinematics_level.name}, {level.name} required; "
                f"call forward_kinematics first")

    # Pinocchio-style aliases (data.py _DEPRECATED_ALIASES)
    @property
    def oMi(self):
        return self.joint_pose_world

    @property
    def oMf(self):
        return self.frame_pose_world

    @property
    def liMi(self):
        return self.joint_pose_local

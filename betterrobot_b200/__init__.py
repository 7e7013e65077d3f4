"""B200-native (sm_100a) batched kinematics and LM-IK path with BetterRobot's call surface.

Public surface (same names as ``better_robot``'s ``src/better_robot/__init__.py:33-44``):
``forward_kinematics``, ``update_frame_placements``, ``compute_joint_jacobians``,
``get_joint_jacobian``, ``get_frame_jacobian``, ``solve_ik`` (+ ``IKCostConfig``,
``OptimizerConfig``, ``IKResult``), ``solve_ik``'s trajectory sibling ``solve_trajopt``,
plus the batched entry points this path adds:
``frame_jacobians`` (fused FK + frame Jacobians), ``solve_ik_batched`` (packed
uneven-batch LM) and ``pose_loss`` (FK pose loss with a hand-written adjoint).
"""

from .data import Data, KinematicsLevel
from .exceptions import (BackendNotAvailableError, BetterRobotError, DeviceMismatchError, DtypeMismatchError,
                         KernelError, QuaternionNormError, ShapeError, StaleCacheError, UnsupportedJointError)
from .ik import BatchIKResult, IKCostConfig, IKResult, OptimizerConfig, PackedIK, solve_ik, solve_ik_batched
from .kinematics import (compute_joint_jacobians, forward_kinematics, frame_jacobians, get_frame_jacobian,
                         get_joint_jacobian, update_frame_placements)
from .model import Frame, JointModel, Model, build_model
from .trajopt import TrajOptConfig, TrajOptResult, solve_trajopt, solve_trajopt_batched

__all__ = [
    "Data", "KinematicsLevel", "Model", "Frame", "JointModel", "build_model",
    "forward_kinematics", "update_frame_placements", "compute_joint_jacobians", "get_joint_jacobian",
    "get_frame_jacobian", "frame_jacobians",
    "solve_ik", "IKCostConfig", "OptimizerConfig", "IKResult", "solve_ik_batched", "PackedIK", "BatchIKResult",
    "solve_trajopt", "solve_trajopt_batched", "TrajOptConfig", "TrajOptResult",
    "BetterRobotError", "BackendNotAvailableError", "DeviceMismatchError", "DtypeMismatchError", "KernelError",
    "QuaternionNormError", "ShapeError", "StaleCacheError", "UnsupportedJointError",
]

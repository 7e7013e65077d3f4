"""Exception classes raised at the Python boundary.

Same names and base classes as ``src/better_robot/exceptions.py:25-131`` so that
code catching BetterRobot's errors keeps working when it calls this path.
``KernelError`` is new: it carries a non-zero status returned by the CUDA library.
"""

from __future__ import annotations


class BetterRobotError(Exception):
    """Root of every exception raised by this package."""


class ModelInconsistencyError(BetterRobotError, ValueError):
    """A ``Model`` violates a topology invariant (parents precede children, contiguous q/v slices)."""


class DeviceMismatchError(BetterRobotError, ValueError):
    """An input tensor lives on a different device than expected (the CUDA path needs CUDA tensors)."""


class DtypeMismatchError(BetterRobotError, ValueError):
    """An input tensor has a dtype the kernels do not accept (they compute in float32)."""


class QuaternionNormError(BetterRobotError, ValueError):
    """A free-flyer quaternion norm is outside ``[0.9, 1.1]``."""


class ShapeError(BetterRobotError, ValueError):
    """A public input has the wrong trailing-axis size."""


class ConvergenceError(BetterRobotError, RuntimeError):
    """Optimizer exited without reaching the requested tolerance (not raised by ``solve_ik``)."""


class BackendNotAvailableError(BetterRobotError, ImportError):
    """The CUDA library could not be loaded, or no CUDA device is present."""


class StaleCacheError(BetterRobotError, RuntimeError):
    """A ``Data`` field was read before the kinematics that fill it ran."""


class UnsupportedJointError(BetterRobotError, ValueError):
    """The model contains a joint kind the device tree table does not encode."""


class KernelError(BetterRobotError, RuntimeError):
    """A C-ABI entry point returned a non-zero status."""

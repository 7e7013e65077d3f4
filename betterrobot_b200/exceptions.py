"""Exception classes raised at the Python boundary.

Same names and base classes as ``src/better_robot/exceptions.py:25-131`` so that
code catching BetterRobot's errors keeps working when it calls this path.  When
BetterRobot itself is importable, every class here also derives from the
reference class of the same name: an error raised by these kernels through the
reference's own entry points (``better_robot.forward_kinematics(...,
backend=BACKEND)``) is caught by ``except better_robot.exceptions.ShapeError``.
``KernelError`` is new: it carries a non-zero status returned by the CUDA library.
"""

from __future__ import annotations

import importlib.util


def _reference_exceptions():
    """BetterRobot's exception module, or None when the package is not installed."""
    try:
        if importlib.util.find_spec("better_robot") is None:
            return None
        from better_robot import exceptions as ref
    except Exception:  # present but not importable (a missing dependency): no reference bases
        return None
    return ref


_REF = _reference_exceptions()


def _bases(name: str, *own: type) -> tuple:
    """``own`` bases, with the reference class ``name`` inserted after this package's root.

    The reference class already derives from its own root and builtin base, so the
    builtin base is dropped when it is present (a consistent method resolution order).
    """
    ref = getattr(_REF, name, None) if _REF is not None else None
    if ref is None:
        return own
    if name == "BetterRobotError":
        return (ref,)
    return tuple(b for b in own if not issubclass(ref, b)) + (ref,)


class BetterRobotError(*_bases("BetterRobotError", Exception)):
    """Root of every exception raised by this package."""


class ModelInconsistencyError(*_bases("ModelInconsistencyError", BetterRobotError, ValueError)):
    """A ``Model`` violates a topology invariant (parents precede children, contiguous q/v slices)."""


class DeviceMismatchError(*_bases("DeviceMismatchError", BetterRobotError, ValueError)):
    """An input tensor lives on a different device than expected (the CUDA path needs CUDA tensors)."""


class DtypeMismatchError(*_bases("DtypeMismatchError", BetterRobotError, ValueError)):
    """An input tensor has a dtype the kernels do not accept (they compute in float32)."""


class QuaternionNormError(*_bases("QuaternionNormError", BetterRobotError, ValueError)):
    """A free-flyer quaternion norm is outside ``[0.9, 1.1]``."""


class ShapeError(*_bases("ShapeError", BetterRobotError, ValueError)):
    """A public input has the wrong trailing-axis size."""


class ConvergenceError(*_bases("ConvergenceError", BetterRobotError, RuntimeError)):
    """Optimizer exited without reaching the requested tolerance (not raised by ``solve_ik``)."""


class BackendNotAvailableError(*_bases("BackendNotAvailableError", BetterRobotError, ImportError)):
    """The CUDA library could not be loaded, or no CUDA device is present."""


class StaleCacheError(*_bases("StaleCacheError", BetterRobotError, RuntimeError)):
    """A ``Data`` field was read before the kinematics that fill it ran."""


class UnsupportedJointError(*_bases("UnsupportedJointError", BetterRobotError, ValueError)):
    """The model contains a joint kind the device tree table does not encode."""


class KernelError(BetterRobotError, RuntimeError):
    """A C-ABI entry point returned a non-zero status (``status``: the code, see ``include/br_b200.h``)."""

    def __init__(self, message: str, status: int = 0):
        super().__init__(message)
        self.status = status

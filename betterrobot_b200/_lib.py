"""ctypes binding of ``libbr_b200.so`` (declarations in ``include/br_b200.h``).

There is no CPU fallback: if the library is missing or no CUDA device is
present, every entry point raises ``BackendNotAvailableError``.
"""

from __future__ import annotations

import ctypes
import os
import threading

from .exceptions import BackendNotAvailableError, KernelError

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbr_b200.so")

c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_void_p = ctypes.c_void_p

STATUS = {0: "ok", -1: "invalid argument", -2: "size above the library limit", -3: "misaligned pointer"}


class BrTree(ctypes.Structure):
    """Mirror of ``br_tree_t``."""

    _fields_ = [("njoints", c_int32), ("nq", c_int32), ("nv", c_int32), ("nframes", c_int32),
                ("rounds", c_int32), ("kinds", c_int32), ("dof_entries", c_int32), ("dof_depth", c_int32),
                ("parent", c_void_p), ("jtype", c_void_p), ("idx_q", c_void_p), ("idx_v", c_void_p),
                ("axis", c_void_p), ("placement", c_void_p), ("support", c_void_p),
                ("frame_parent", c_void_p), ("frame_placement", c_void_p),
                ("col_joint", c_void_p), ("col_kind", c_void_p), ("col_axis", c_void_p),
                ("lower", c_void_p), ("upper", c_void_p), ("dof_sched", c_void_p)]


class IKSettings(ctypes.Structure):
    _fields_ = [("lam0", ctypes.c_float), ("factor", ctypes.c_float), ("tol", ctypes.c_float),
                ("lam_min", ctypes.c_float), ("lam_max", ctypes.c_float), ("gn_eps", ctypes.c_float),
                ("pos_weight", ctypes.c_float), ("ori_weight", ctypes.c_float),
                ("limit_weight", ctypes.c_float), ("rest_weight", ctypes.c_float),
                ("max_iter", c_int32), ("optimizer", c_int32), ("kernel", c_int32),
                ("kernel_param", ctypes.c_float), ("precision", c_int32)]


class IKBatch(ctypes.Structure):
    _fields_ = [("n_problems", c_int32), ("max_targets", c_int32), ("n_classes", c_int32), ("n_items", c_int32),
                ("trees", ctypes.POINTER(BrTree)), ("team_size", ctypes.POINTER(c_int32)),
                ("items", c_void_p), ("order", c_void_p), ("n_targets", c_void_p), ("frames", c_void_p),
                ("targets", c_void_p), ("q_offset", c_void_p), ("x0", c_void_p), ("q_rest", c_void_p),
                ("r_offset", c_void_p), ("target_kind", c_void_p)]


class IKResultBuf(ctypes.Structure):
    _fields_ = [("x", c_void_p), ("iters", c_void_p), ("status", c_void_p), ("cost", c_void_p),
                ("residual", c_void_p)]


class TrajSettings(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("w_goal", ctypes.c_float), ("w_start", ctypes.c_float),
                ("w_accel", ctypes.c_float), ("w_limit", ctypes.c_float), ("w_ref", ctypes.c_float),
                ("tol", ctypes.c_float), ("gn_eps", ctypes.c_float), ("lam0", ctypes.c_float),
                ("factor", ctypes.c_float), ("lam_min", ctypes.c_float), ("lam_max", ctypes.c_float),
                ("max_iter", c_int32), ("optimizer", c_int32)]


# name -> (restype, argtypes); must match include/br_b200.h
SIGNATURES: dict[str, tuple] = {
    "br_version": (ctypes.c_char_p, []),
    "br_forward_kinematics": (c_int32, [ctypes.POINTER(BrTree), c_void_p, c_int64, c_void_p, c_void_p,
                                        c_void_p, c_int32, c_void_p, c_void_p]),
    "br_frame_jacobians": (c_int32, [ctypes.POINTER(BrTree), c_void_p, c_int64, c_void_p, c_int32, c_int32,
                                     c_void_p, c_void_p, c_void_p]),
    "br_frame_jacobians_from_poses": (c_int32, [ctypes.POINTER(BrTree), c_void_p, c_int64, c_void_p, c_int32,
                                                c_int32, c_void_p, c_void_p]),
    "br_lm_solve": (c_int32, [ctypes.POINTER(IKBatch), ctypes.POINTER(IKSettings), ctypes.POINTER(IKResultBuf),
                              c_int32, c_void_p, c_int64, c_void_p]),
    "br_lm_team_floats": (c_int64, [ctypes.POINTER(BrTree), c_int32]),
    "br_dof_schedule": (c_int64, [c_void_p, c_int32, c_void_p, c_int64]),
    "br_lm_solve_noalloc": (c_int32, [ctypes.POINTER(IKBatch), ctypes.POINTER(IKSettings),
                                      ctypes.POINTER(IKResultBuf), c_int32, c_void_p]),
    "br_trajopt_solve": (c_int32, [ctypes.POINTER(BrTree), c_int32, c_int64, c_int32, c_void_p, c_void_p, c_void_p,
                                   c_void_p, ctypes.POINTER(TrajSettings), c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p]),
    "br_configuration_op": (c_int32, [ctypes.POINTER(BrTree), c_void_p, c_int32, c_int32, c_void_p, c_void_p,
                                      c_int64, c_void_p, c_void_p]),
    "br_lie_op": (c_int32, [c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p]),
    "br_lie_op_sizes": (c_int32, [c_int32, c_void_p, c_void_p, c_void_p]),
    "br_pose_loss": (c_int32, [ctypes.POINTER(BrTree), c_void_p, c_int64, c_void_p, c_int32, c_void_p, c_void_p,
                               c_int32, c_void_p, c_void_p, c_void_p]),
    "br_pose_loss_backward": (c_int32, [ctypes.POINTER(BrTree), c_void_p, c_void_p, c_int64, c_void_p, c_int32,
                                        c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
}

_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH):
    """Load the shared library (no device is touched)."""
    global _lib
    if _lib is not None:  # loaded: no lock on the per-call path
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise BackendNotAvailableError(
                    f"{path} is missing; build it with `python -m betterrobot_b200.build` (nvcc, sm_100a)")
            lib = ctypes.CDLL(path)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def call(name: str, *args) -> None:
    """Call an entry point and raise ``KernelError`` on a non-zero status."""
    st = getattr(load(), name)(*args)
    if st != 0:
        msg = STATUS.get(st, f"CUDA error {st}")
        raise KernelError(f"{name} returned {st} ({msg})", st)


_cuda_seen = False


def require_cuda(t) -> None:
    global _cuda_seen
    if not _cuda_seen:  # a device, once found, stays for the process
        import torch
        if not torch.cuda.is_available():
            raise BackendNotAvailableError("the sm_100a path needs a CUDA device; none is available")
        _cuda_seen = True
    if not t.is_cuda:
        from .exceptions import DeviceMismatchError
        raise DeviceMismatchError(f"expected a CUDA tensor, got device={t.device}")


def stream_ptr(device=None) -> int:
    import torch
    return torch.cuda.current_stream(device).cuda_stream

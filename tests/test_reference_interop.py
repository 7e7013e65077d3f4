"""Drop-in checks against BetterRobot itself, on the CPU (no kernel runs).

* A ``Model`` built by the reference's own ``ModelBuilder`` + ``build_model`` packs into
  exactly the same device tree table as this package's ``Model`` of the same robot.
* ``B200Backend`` satisfies the reference's runtime-checkable ``Backend`` Protocols
  (``src/better_robot/backends/protocol.py:27-119``).
* The reference's public ``forward_kinematics(..., backend=BACKEND)`` dispatches into this
  package (on a machine without a GPU the call stops at the CUDA check).

Runs where BetterRobot is importable: its source tree named by ``BETTERROBOT_SRC`` (the
directory that holds the ``better_robot`` package), or an installed ``better_robot``.
Elsewhere every test here is skipped.
"""

import importlib.util
import os
import sys

import numpy as np
import pytest
import torch

SRC = os.environ.get("BETTERROBOT_SRC")
if SRC and os.path.isdir(os.path.join(SRC, "better_robot")) and SRC not in sys.path:
    sys.path.insert(0, SRC)
HAVE_REFERENCE = importlib.util.find_spec("better_robot") is not None
pytestmark = pytest.mark.skipif(not HAVE_REFERENCE, reason="BetterRobot is not importable (set BETTERROBOT_SRC)")
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))

from betterrobot_b200 import synthetic as syn  # noqa: E402
from betterrobot_b200.tree import TreeArrays  # noqa: E402

SPECS = {"chain7": syn.chain_spec(), "humanoid": syn.humanoid_spec(), "dual_arm": syn.dual_arm_spec()}


@pytest.mark.parametrize("name", list(SPECS))
def test_reference_model_packs_identically(name):
    from make_golden import reference_model
    ref = reference_model(SPECS[name])
    mine = syn.model_from_spec(SPECS[name], dtype=torch.float64)
    a, b = TreeArrays(ref), TreeArrays(mine)
    assert (a.nj, a.nq, a.nv, a.nf, a.rounds) == (b.nj, b.nq, b.nv, b.nf, b.rounds)
    for (na, xa), (nb, xb) in zip(a.sections(), b.sections()):
        assert na == nb
        np.testing.assert_array_equal(xa, xb, err_msg=na)


def test_backend_satisfies_reference_protocols():
    from better_robot.backends.protocol import Backend, DynamicsOps, KinematicsOps, LieOps
    from betterrobot_b200.backend import BACKEND
    assert isinstance(BACKEND, Backend)
    assert isinstance(BACKEND.lie, LieOps)
    assert isinstance(BACKEND.kinematics, KinematicsOps)
    assert isinstance(BACKEND.dynamics, DynamicsOps)


def test_reference_entry_point_dispatches_here():
    import better_robot as br_ref
    from make_golden import reference_model
    from betterrobot_b200.backend import BACKEND
    from betterrobot_b200.exceptions import BetterRobotError
    if torch.cuda.is_available():
        pytest.skip("CPU-only check")
    m = reference_model(SPECS["chain7"])
    q = torch.zeros(2, m.nq, dtype=torch.float32)
    with pytest.raises(BetterRobotError, match="CUDA"):
        br_ref.forward_kinematics(m, q, backend=BACKEND)


def test_reference_except_clauses_catch_errors_raised_here():
    """With BetterRobot importable, this package's exception classes derive from the reference's:
    an error raised by these kernels through the reference's own entry point is caught by
    ``except better_robot.exceptions.<Name>``.  Run in a fresh interpreter so that the import
    order (reference first or not) is the one a user has."""
    import subprocess
    import textwrap
    code = textwrap.dedent("""
        import sys, torch
        import better_robot as br_ref
        from better_robot import exceptions as rex
        from betterrobot_b200 import exceptions as ex
        from betterrobot_b200.backend import BACKEND
        from make_golden import reference_model
        from betterrobot_b200 import synthetic as syn
        names = ["BetterRobotError", "ModelInconsistencyError", "DeviceMismatchError", "DtypeMismatchError",
                 "QuaternionNormError", "ShapeError", "ConvergenceError", "BackendNotAvailableError",
                 "StaleCacheError", "UnsupportedJointError"]
        for n in names:
            assert issubclass(getattr(ex, n), getattr(rex, n)), n
            assert issubclass(getattr(ex, n), ex.BetterRobotError), n
        assert issubclass(ex.KernelError, rex.BetterRobotError)
        m = reference_model(syn.chain_spec())
        q = torch.zeros(2, m.nq, dtype=torch.float32)   # a CPU tensor: this backend refuses it
        try:
            br_ref.forward_kinematics(m, q, backend=BACKEND)
        except rex.BetterRobotError as e:
            assert isinstance(e, ex.BetterRobotError), type(e)
            print("caught", type(e).__name__)
        else:
            raise SystemExit("no error raised")
    """)
    here = os.path.dirname(os.path.abspath(__file__))
    path = [p for p in (SRC, os.path.dirname(here), os.path.join(here, "golden")) if p]
    env = dict(os.environ, PYTHONPATH=os.pathsep.join(path + [os.environ.get("PYTHONPATH", "")]),
               CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caught" in r.stdout


def test_solve_trajopt_reads_reference_cost_stack():
    """The solve_trajopt facade reads a CostStack built from BetterRobot's own residual classes
    (the stack of ``tasks/trajopt.py``'s docstring and of the golden solves) into the kernel's
    weights and targets."""
    import torch as _t
    from better_robot.costs.stack import CostStack
    from better_robot.optim.optimizers.gauss_newton import GaussNewton
    from better_robot.residuals import AccelerationResidual, JointPositionLimit, PoseResidual, TimeIndexedResidual
    from better_robot.residuals.regularization import ReferenceTrajectoryResidual
    from make_golden import reference_model
    from betterrobot_b200.trajopt import _stack_to_config
    m = reference_model(SPECS["chain7"])
    T = 8
    X0 = _t.zeros(T, m.nq, dtype=_t.float64)
    Tg = _t.tensor([0.1, 0.2, 0.3, 0.0, 0.0, 0.0, 1.0], dtype=_t.float64)
    Ts = _t.tensor([0.0, 0.2, 0.3, 0.0, 0.0, 0.0, 1.0], dtype=_t.float64)
    fid = m.frame_id("ee")
    st = CostStack()
    st.add("goal", TimeIndexedResidual(PoseResidual(frame_id=fid, target=Tg), t_idx=T - 1), weight=2.0)
    st.add("start", TimeIndexedResidual(PoseResidual(frame_id=fid, target=Ts), t_idx=0), weight=0.5)
    st.add("accel", AccelerationResidual(m, dt=0.1), weight=1e-2)
    for t in range(T):
        st.add(f"limits_t{t}", TimeIndexedResidual(JointPositionLimit(m), t_idx=t, name=f"limits_t{t}"), weight=0.1)
    st.add("ref", ReferenceTrajectoryResidual(m, X0.clone()), weight=1e-3)
    cfg, f, goal, start, q_ref = _stack_to_config(m, st, T, GaussNewton(tol=1e-7), 40)
    assert f == fid and _t.equal(goal, Tg) and _t.equal(start, Ts) and _t.equal(q_ref, X0)
    assert (cfg.w_goal, cfg.w_start, cfg.w_accel, cfg.w_limit, cfg.w_ref) == (2.0, 0.5, 1e-2, 0.1, 1e-3)
    assert (cfg.dt, cfg.optimizer, cfg.tol, cfg.max_iter) == (0.1, "gn", 1e-7, 40)
    st.set_active("ref", False)
    assert _stack_to_config(m, st, T, GaussNewton(), 40)[0].w_ref == 0.0

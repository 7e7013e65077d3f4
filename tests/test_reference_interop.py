"""Drop-in checks against BetterRobot itself, on the CPU (no kernel runs).

* A ``Model`` built by the reference's own ``ModelBuilder`` + ``build_model`` packs into
  exactly the same device tree table as this package's ``Model`` of the same robot.
* ``B200Backend`` satisfies the reference's runtime-checkable ``Backend`` Protocols
  (``src/better_robot/backends/protocol.py:27-119``).
* The reference's public ``forward_kinematics(..., backend=BACKEND)`` dispatches into this
  package (on a machine without a GPU the call stops at the CUDA check).

Skipped where the reference source tree is not present (``BETTERROBOT_SRC``).
"""

import os
import sys

import numpy as np
import pytest
import torch

SRC = os.environ.get("BETTERROBOT_SRC", "/root/reference/src")
if not os.path.isdir(os.path.join(SRC, "better_robot")):
    pytest.skip("BetterRobot source tree not available", allow_module_level=True)
sys.path.insert(0, SRC)
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))

from betterrobot_b200 import synthetic as syn  # noqa: E402
from betterrobot_b200.backend import BACKEND  # noqa: E402
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
    assert isinstance(BACKEND, Backend)
    assert isinstance(BACKEND.lie, LieOps)
    assert isinstance(BACKEND.kinematics, KinematicsOps)
    assert isinstance(BACKEND.dynamics, DynamicsOps)


def test_reference_entry_point_dispatches_here():
    import better_robot as br_ref
    from make_golden import reference_model
    from betterrobot_b200.exceptions import BetterRobotError
    if torch.cuda.is_available():
        pytest.skip("CPU-only check")
    m = reference_model(SPECS["chain7"])
    q = torch.zeros(2, m.nq, dtype=torch.float32)
    with pytest.raises(BetterRobotError, match="CUDA"):
        br_ref.forward_kinematics(m, q, backend=BACKEND)

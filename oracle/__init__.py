"""CPU oracle for the kinematics + LM-IK path — TEST INFRASTRUCTURE ONLY.

A float64 numpy restatement of BetterRobot's own torch implementation of the
path (each function cites the reference ``file:line`` it follows).  It is the
checker for the CUDA library: only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg (``cpu_baseline`` / ``--impl reference``) may
import it.  The product path never calls into this package.

Parity of the oracle itself is pinned by ``tests/golden/*.npz``: outputs of the
reference (``better_robot`` v0.2.0, torch 2.11.0) run in float64 on the same
seeded inputs, generated by ``tests/golden/make_golden.py``.
"""

"""The Python host code's copies of the C ABI's constants equal the header's ``#define``s
(``include/br_b200.h``): joint kinds, reference frames, limits, operation, optimizer,
kernel, precision and target-kind codes, and the Lie op table.  Read from the header text,
so no device and no library call is needed."""

import os
import re

import pytest

from betterrobot_b200 import autotune, configuration, ik, kinematics, lie, tree

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "br_b200.h")


@pytest.fixture(scope="module")
def defines():
    out = {}
    with open(HEADER) as f:
        for line in f:
            m = re.match(r"#define\s+(BR_\w+)\s+\(?(-?\d+)\)?", line)
            if m:
                out[m.group(1)] = int(m.group(2))
    return out


def test_joint_kinds_and_tree_limits(defines):
    assert (tree.JOINT_FIXED, tree.JOINT_REVOLUTE, tree.JOINT_PRISMATIC, tree.JOINT_FREE_FLYER,
            tree.JOINT_SPHERICAL, tree.JOINT_PLANAR, tree.JOINT_REVOLUTE_UNBOUNDED, tree.JOINT_TRANSLATION) == tuple(
        defines[f"BR_JOINT_{k}"] for k in ("FIXED", "REVOLUTE", "PRISMATIC", "FREE_FLYER", "SPHERICAL", "PLANAR",
                                           "REVOLUTE_UNBOUNDED", "TRANSLATION"))
    assert (tree.MAX_JOINTS, tree.MAX_NV, tree.MAX_NQ) == (defines["BR_MAX_JOINTS"], defines["BR_MAX_NV"],
                                                            defines["BR_MAX_NQ"])


def test_reference_frames_and_configuration_ops(defines):
    assert kinematics._REF == {"world": defines["BR_REF_WORLD"],
                               "local_world_aligned": defines["BR_REF_LOCAL_WORLD_ALIGNED"],
                               "local": defines["BR_REF_LOCAL"]}
    assert (configuration.OP_INTEGRATE, configuration.OP_DIFFERENCE) == (defines["BR_OP_INTEGRATE"],
                                                                          defines["BR_OP_DIFFERENCE"])


def test_ik_codes_and_limits(defines):
    assert (ik.MAX_CLASSES, ik.MAX_TARGETS) == (defines["BR_MAX_IK_CLASSES"], defines["BR_MAX_IK_TARGETS"])
    assert (ik.OPT_LM, ik.OPT_GN) == (defines["BR_OPT_LM"], defines["BR_OPT_GN"])
    assert ik.KERNELS == {k: defines[f"BR_KERNEL_{k.upper()}"] for k in ("l2", "huber", "cauchy", "tukey")}
    assert ik.PRECISIONS == {"f32": defines["BR_PREC_F32"], "f64": defines["BR_PREC_F64"]}
    assert ik.TARGET_KINDS == {k: defines[f"BR_TARGET_{k.upper()}"] for k in ("pose", "position", "orientation")}
    assert autotune.BR_ETOOBIG == defines["BR_ETOOBIG"]


def test_lie_op_codes(defines):
    c_name = {"right_jacobian_se3": "SE3_JR", "right_jacobian_inv_se3": "SE3_JR_INV"}
    for name, code in lie.OPS.items():
        assert defines["BR_LIE_" + c_name.get(name, name.upper())] == code, name
    assert len(lie.OPS) == len([k for k in defines if k.startswith("BR_LIE_")])

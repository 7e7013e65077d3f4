"""The benchmark's workload definition on the CPU: the seeded 8,192-problem uneven IK mix is
reproducible, has the stated class shares and target counts, and ranks get disjoint seeds;
the FLOP accounting behind the bench line's compute rooflines is positive and grows with the
work it counts."""

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))

import bench  # noqa: E402
from betterrobot_b200 import synthetic as syn  # noqa: E402


def test_uneven_mix_shares_and_targets():
    mix = syn.ik_uneven_mix(bench.N_PROBLEMS, bench.shard_seed(0))
    labels = [lab for lab, _ in mix]
    assert len(mix) == 8192
    assert (labels.count("chain7"), labels.count("dual_arm"), labels.count("humanoid")) == (3277, 2458, 2457)
    kt = np.array([k for _, k in mix])
    assert kt.min() == 1 and kt.max() == 6
    assert mix == syn.ik_uneven_mix(bench.N_PROBLEMS, bench.shard_seed(0))   # seeded
    assert mix != syn.ik_uneven_mix(bench.N_PROBLEMS, bench.shard_seed(1))   # another rank's set


def test_workload_is_reproducible():
    a = bench.make_workload(256, bench.shard_seed(0))
    b = bench.make_workload(256, bench.shard_seed(0))
    assert [c["name"] for c in a] == ["humanoid", "dual_arm", "chain7"]
    for ca, cb in zip(a, b):
        np.testing.assert_array_equal(ca["frames"], cb["frames"])
        np.testing.assert_array_equal(ca["n_targets"], cb["n_targets"])
        np.testing.assert_array_equal(ca["q0"].numpy(), cb["q0"].numpy())
        # every problem's targets are distinct candidate frames of its robot
        assert all(len(set(r)) == 6 for r in ca["frames"].tolist())
    assert sum(len(c["n_targets"]) for c in a) == 256


def test_flop_accounting():
    assert bench.FP32_PEAK_TFLOPS > 70
    m = syn.model_from_spec(syn.humanoid_spec())
    fids = syn.op_frame_ids(m)
    f1 = bench.adjoint_flops_per_config(m, fids, recompute=False)
    f2 = bench.adjoint_flops_per_config(m, fids, recompute=True)
    assert 0 < f1 < f2
    assert 0 < bench.lm_iteration_flops(m, fids[:1]) < bench.lm_iteration_flops(m, fids[:6])

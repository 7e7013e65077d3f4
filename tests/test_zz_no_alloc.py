"""br_lm_solve_noalloc: the allocation-free LM entry point, called through the C ABI.

This entry point serves callers that cannot allocate device memory (a real-time
controller loop, a host without a CUDA allocator): its 16-byte work-queue
scratch comes from a static device array inside the library instead of a caller
buffer.  The test solves one uneven batch with br_lm_solve, then twice in a row
with br_lm_solve_noalloc into separate output buffers, and requires the same
answers each time (the second call also checks that the shared scratch is
cleared before reuse).  Tolerance: solutions within 1e-5 (the kernels are the
same, so they agree exactly in practice); iterations and status identical.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _batch():
    from betterrobot_b200 import ik as bik, synthetic as syn
    import betterrobot_b200 as br
    specs = [syn.humanoid_spec(), syn.dual_arm_spec(), syn.chain_spec()]
    cand = [[f"track{i}" for i in range(4)], ["ee_l", "ee_r", "body_l_link5", "body_r_link5"],
            ["ee", "body_link7", "body_link5", "body_link3"]]
    rng = np.random.default_rng(11)
    models, frames, nts, tg, q0s = [], [], [], [], []
    for spec, names in zip(specs, cand):
        m = syn.model_from_spec(spec)
        m64 = syn.model_from_spec(spec, dtype=torch.float64)
        P = 40
        fids = np.array([m.frame_id(n) for n in names], np.int32)
        q_star = syn.random_q(m64, P, 12, rev_range=2.5, base_translation=0.5)
        d = br.forward_kinematics(m, q_star.float().cuda(), compute_frames=True)
        models.append(m)
        frames.append(np.broadcast_to(fids, (P, len(fids))))
        nts.append(rng.integers(1, len(fids) + 1, size=P).astype(np.int32))
        tg.append(d.frame_pose_world[:, torch.from_numpy(fids).long().cuda()].contiguous())
        q0s.append(syn.noisy_start(m64, q_star, 0.3, 13).float().cuda())
    pk = bik.PackedIK(models, frames, nts)
    pk.set_inputs(tg, q0s)
    settings = bik.settings_from(bik.IKCostConfig(rest_weight=1e-3),
                                 bik.OptimizerConfig(max_iter=60, lam0=1e-3, factor=10.0))
    return pk, settings


def test_noalloc_entry_point_matches_allocating_one_twice():
    from betterrobot_b200 import _lib
    lib = _lib.load()
    pk, settings = _batch()
    pk.solve(settings)
    torch.cuda.synchronize()
    ref = (pk.x.clone(), pk.iters.clone(), pk.status.clone(), pk.cost.clone())
    x = torch.empty_like(pk.x)
    iters = torch.empty_like(pk.iters)
    status = torch.empty_like(pk.status)
    cost = torch.empty_like(pk.cost)
    res = _lib.IKResultBuf()
    res.x, res.iters, res.status, res.cost = x.data_ptr(), iters.data_ptr(), status.data_ptr(), cost.data_ptr()
    res.residual = None
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        x.fill_(float("nan"))
        iters.fill_(-1)
        status.fill_(-1)
        cost.fill_(float("nan"))
        st = lib.br_lm_solve_noalloc(ctypes.byref(pk._batch), ctypes.byref(settings), ctypes.byref(res),
                                     pk.warps_per_cta, stream)
        assert st == 0, f"call {call}: status {st}"
        torch.cuda.synchronize()
        torch.testing.assert_close(x, ref[0], rtol=0, atol=1e-5)
        assert torch.equal(iters, ref[1]), call
        assert torch.equal(status, ref[2]), call
        torch.testing.assert_close(cost, ref[3], rtol=1e-6, atol=1e-9)


def test_noalloc_rejects_bad_arguments():
    from betterrobot_b200 import _lib
    lib = _lib.load()
    pk, settings = _batch()
    res = _lib.IKResultBuf()
    assert lib.br_lm_solve_noalloc(None, ctypes.byref(settings), ctypes.byref(res), 4, None) == -1
    assert lib.br_lm_solve_noalloc(ctypes.byref(pk._batch), ctypes.byref(settings), ctypes.byref(res), 4, None) == -1

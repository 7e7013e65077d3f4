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


def _batch(classes=(0, 1, 2), warps_per_cta=4):
    from betterrobot_b200 import ik as bik, synthetic as syn
    import betterrobot_b200 as br
    specs = [syn.humanoid_spec(), syn.dual_arm_spec(), syn.chain_spec()]
    cand = [[f"track{i}" for i in range(4)], ["ee_l", "ee_r", "body_l_link5", "body_r_link5"],
            ["ee", "body_link7", "body_link5", "body_link3"]]
    specs = [specs[c] for c in classes]
    cand = [cand[c] for c in classes]
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
    pk = bik.PackedIK(models, frames, nts, warps_per_cta=warps_per_cta)
    pk.set_inputs(tg, q0s)
    settings = bik.settings_from(bik.IKCostConfig(rest_weight=1e-3),
                                 bik.OptimizerConfig(max_iter=60, lam0=1e-3, factor=10.0))
    return pk, settings


def _noalloc_outputs(pk):
    from betterrobot_b200 import _lib
    x = torch.empty_like(pk.x)
    iters = torch.empty_like(pk.iters)
    status = torch.empty_like(pk.status)
    cost = torch.empty_like(pk.cost)
    res = _lib.IKResultBuf()
    res.x, res.iters, res.status, res.cost = x.data_ptr(), iters.data_ptr(), status.data_ptr(), cost.data_ptr()
    res.residual = None
    return (x, iters, status, cost), res


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


def test_allocating_launch_after_smaller_noalloc_launch():
    """A large br_lm_solve launch, then a small br_lm_solve_noalloc launch (chains only, one warp
    per CTA: less shared memory), then a br_lm_solve launch whose shared memory lies between the
    two.  The entry points share one record of the shared memory each kernel is allowed, so the
    third launch must still start; its results must equal the allocation-free solve of the same
    batch."""
    from betterrobot_b200 import _lib
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    big, settings = _batch((0, 1, 2), warps_per_cta=8)
    big.solve(settings)
    small, _ = _batch((2,), warps_per_cta=1)
    out_s, res_s = _noalloc_outputs(small)
    assert lib.br_lm_solve_noalloc(ctypes.byref(small._batch), ctypes.byref(settings), ctypes.byref(res_s),
                                   1, stream) == 0
    mid, _ = _batch((1,), warps_per_cta=8)
    mid.solve(settings)  # raises KernelError on a failed launch
    torch.cuda.synchronize()
    out_m, res_m = _noalloc_outputs(mid)
    assert lib.br_lm_solve_noalloc(ctypes.byref(mid._batch), ctypes.byref(settings), ctypes.byref(res_m),
                                   mid.warps_per_cta, stream) == 0
    torch.cuda.synchronize()
    torch.testing.assert_close(out_m[0], mid.x, rtol=0, atol=1e-5)
    assert torch.equal(out_m[1], mid.iters) and torch.equal(out_m[2], mid.status)
    assert bool(((out_s[2] & 0xFF) <= 1).all())  # every chain problem ended: converged or at the iteration limit


def test_noalloc_rejects_bad_arguments():
    from betterrobot_b200 import _lib
    lib = _lib.load()
    pk, settings = _batch()
    res = _lib.IKResultBuf()
    assert lib.br_lm_solve_noalloc(None, ctypes.byref(settings), ctypes.byref(res), 4, None) == -1
    assert lib.br_lm_solve_noalloc(ctypes.byref(pk._batch), ctypes.byref(settings), ctypes.byref(res), 4, None) == -1

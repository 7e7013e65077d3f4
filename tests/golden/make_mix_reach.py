"""Per-problem outcome of the float64 oracle LM on the whole 8,192-problem IK mix of
``bench.py`` (same workload, seed 7, same settings): ``ik_mix_reach.npz`` with, per problem,
its class, index in the class, whether every target ends within 1e-4 m / 1e-4 rad, the
converged flag and the iteration count.  The oracle is pinned to the reference's own
solves (``test_oracle_golden.py``); this fixture carries it to the full benchmark size.

    python tests/golden/make_mix_reach.py          # ~10 CPU-minutes on 8 processes
"""

import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _chunk(args):
    import torch
    torch.set_num_threads(1)
    import bench
    from oracle import ik as oik, kinematics as K
    ci, lo, hi = args
    c = bench.make_workload(bench.N_PROBLEMS, 7)[ci]
    m64 = c["model64"]
    s = oik.IKSettings(lam0=bench.SETTINGS["lam0"], factor=bench.SETTINGS["factor"], tol=bench.SETTINGS["tol"],
                       max_iter=bench.MAX_ITER, rest_weight=bench.SETTINGS["rest_weight"],
                       limit_weight=bench.SETTINGS["limit_weight"])
    rows = []
    for p in range(lo, hi):
        k = int(c["n_targets"][p])
        fids = [int(f) for f in c["frames"][p, :k]]
        oMi, _ = K.forward_kinematics(m64, c["q_star"].numpy()[p:p + 1])
        T = K.frame_placements(m64, oMi, fids)
        r = oik.solve(m64, fids, T, c["q0"].numpy()[p:p + 1], s)
        pe, re = oik.pose_errors(m64, r.q, fids, T)
        rows.append((ci, p, int(pe[0] <= bench.REACH_TOL and re[0] <= bench.REACH_TOL), int(r.converged[0]),
                     int(r.iters[0])))
    return rows


def main():
    import bench
    wl = bench.make_workload(bench.N_PROBLEMS, 7)
    jobs = [(ci, lo, min(len(c["n_targets"]), lo + 64)) for ci, c in enumerate(wl)
            for lo in range(0, len(c["n_targets"]), 64)]
    with mp.get_context("spawn").Pool(int(os.environ.get("PROCS", "8"))) as pool:
        rows = [r for chunk in pool.imap_unordered(_chunk, jobs) for r in chunk]
    a = np.array(sorted(rows), np.int16)
    np.savez_compressed(os.path.join(HERE, "ik_mix_reach.npz"), cls=a[:, 0], index=a[:, 1], reached=a[:, 2],
                        converged=a[:, 3], iters=a[:, 4], classes=np.array([c["name"] for c in wl]))
    print("reached", int(a[:, 2].sum()), "converged", int(a[:, 3].sum()), "of", len(a))


if __name__ == "__main__":
    main()

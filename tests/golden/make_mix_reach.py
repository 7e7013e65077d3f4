"""Per-problem outcome of the float64 oracle LM on the whole 8,192-problem IK mix of
``bench.py`` (same workload, seed 7, same settings), and of BetterRobot's own float64 LM
on the same problems: ``ik_mix_reach.npz`` with, per problem,

* ``cls``, ``index``: its class and index in the class;
* ``reached``: every target ends within 1e-4 m / 1e-4 rad (oracle);
* ``converged``, ``iters``: the oracle's verdict and iteration count;
* ``margin``: the oracle's smallest ``|cost_new - cost|`` in units of the cost's float64
  spacing over the accept tests that decide convergence (``oracle.ik.IKOutcome.margin``);
  a verdict with a margin of a few units is decided by the rounding of a float64 sum;
* ``q_final`` (packed per problem in class order, ``q_offset``), ``cost``: the oracle's final
  configuration and ``0.5 |r|^2``;
* ``ref_converged``, ``ref_iters``: the verdict and iteration count of BetterRobot's
  ``LevenbergMarquardt`` run in float64 through its own cost stack (the solve of
  ``make_golden.reference_lm``, built as ``solve_ik`` builds it).

The oracle is pinned to the reference's own solves (``test_oracle_golden.py``); this fixture
carries the comparison to the full benchmark size.

    BETTERROBOT_SRC=<reference>/src python tests/golden/make_mix_reach.py   # ~1 h on 8 processes
"""

import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def _chunk(args):
    import torch
    torch.set_num_threads(1)
    import bench
    from oracle import ik as oik, kinematics as K
    ci, lo, hi = args
    name, spec = bench.class_specs()[ci]
    c = bench.make_workload(bench.N_PROBLEMS, 7)[ci]
    m64 = c["model64"]
    s = oik.IKSettings(lam0=bench.SETTINGS["lam0"], factor=bench.SETTINGS["factor"], tol=bench.SETTINGS["tol"],
                       max_iter=bench.MAX_ITER, rest_weight=bench.SETTINGS["rest_weight"],
                       limit_weight=bench.SETTINGS["limit_weight"])
    src = os.environ.get("BETTERROBOT_SRC")
    if src:
        sys.path.insert(0, src)
    from make_golden import reference_lm, reference_model
    from better_robot.kinematics.forward import forward_kinematics as ref_fk
    mref = reference_model(spec)
    rows = []
    for p in range(lo, hi):
        k = int(c["n_targets"][p])
        fids = [int(f) for f in c["frames"][p, :k]]
        oMi, _ = K.forward_kinematics(m64, c["q_star"].numpy()[p:p + 1])
        T = K.frame_placements(m64, oMi, fids)
        r = oik.solve(m64, fids, T, c["q0"].numpy()[p:p + 1], s)
        pe, re = oik.pose_errors(m64, r.q, fids, T)
        names = [c["model"].frames[f].name for f in fids]
        d = ref_fk(mref, c["q_star"][p:p + 1].double(), compute_frames=True)
        Tref = d.frame_pose_world[0, [mref.frame_id(n) for n in names], :].clone()
        st = reference_lm(mref, names, Tref, c["q0"][p].double(), tol=s.tol, max_iter=s.max_iter, lam0=s.lam0,
                          factor=s.factor, limit_w=s.limit_weight, rest_w=s.rest_weight)
        rows.append((ci, p, int(pe[0] <= bench.REACH_TOL and re[0] <= bench.REACH_TOL), int(r.converged[0]),
                     int(r.iters[0]), float(r.margin[0]), int(st.status == "converged"), int(st.iters),
                     r.q[0].copy(), float(r.cost[0])))
    return rows


def main():
    import bench
    if not os.environ.get("BETTERROBOT_SRC"):
        raise SystemExit("set BETTERROBOT_SRC to the reference's src directory")
    wl = bench.make_workload(bench.N_PROBLEMS, 7)
    jobs = [(ci, lo, min(len(c["n_targets"]), lo + 32)) for ci, c in enumerate(wl)
            for lo in range(0, len(c["n_targets"]), 32)]
    jobs.sort(key=lambda j: j[0])  # humanoid chunks (the slowest) first
    with mp.get_context("spawn").Pool(int(os.environ.get("PROCS", "8"))) as pool:
        rows = sorted((r for chunk in pool.imap_unordered(_chunk, jobs) for r in chunk), key=lambda r: (r[0], r[1]))
    a = np.array([r[:5] for r in rows], np.int16)
    qf = [r[8] for r in rows]
    q_offset = np.concatenate([[0], np.cumsum([len(x) for x in qf])[:-1]]).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "ik_mix_reach.npz"), cls=a[:, 0], index=a[:, 1], reached=a[:, 2],
                        converged=a[:, 3], iters=a[:, 4], margin=np.array([r[5] for r in rows], np.float32),
                        q_final=np.concatenate(qf), q_offset=q_offset, cost=np.array([r[9] for r in rows]),
                        ref_converged=np.array([r[6] for r in rows], np.int8),
                        ref_iters=np.array([r[7] for r in rows], np.int16),
                        classes=np.array([c["name"] for c in wl]))
    print("reached", int(a[:, 2].sum()), "converged", int(a[:, 3].sum()), "of", len(a),
          "reference converged", sum(r[6] for r in rows))


if __name__ == "__main__":
    main()

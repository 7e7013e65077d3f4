// traj_gn.cu — batched trajectory optimisation (Gauss-Newton / LM) with a
// block-banded Cholesky, one warp per trajectory.
//
// Reference: solve_trajopt with knot parameterisation
// (src/better_robot/tasks/trajopt.py:84-230) flattens a (T, nq) trajectory into one
// least-squares problem and solves the dense (T*nv)^2 normal equations with a
// dense Cholesky every iteration (448 x 448 for T = 64, nv = 7).  The stack here is
//   goal  : PoseResidual at knot T-1        (TimeIndexedResidual, residuals/temporal.py:20-126)
//   start : PoseResidual at knot 0          (optional)
//   accel : (q_{s+2} - 2 q_{s+1} + q_s)/dt^2 (AccelerationResidual, residuals/smoothness.py:98-161)
//   limits: JointPositionLimit at every knot (residuals/limits.py:56-86)
//   ref   : q_t - q_ref_t                   (ReferenceTrajectoryResidual, residuals/regularization.py:133-152)
// each with a CostStack item weight.  Its J^T J is block PENTA-diagonal in 7x7
// blocks (the acceleration row couples three knots), with the acceleration part a
// scalar band times I: this kernel assembles only the bands — H_tt, H_{t+1,t},
// H_{t+2,t} — and factors them with a bandwidth-2 block Cholesky
//   L_tt     = chol(H_tt - L_{t,t-1} L_{t,t-1}^T - L_{t,t-2} L_{t,t-2}^T)
//   L_{t+1,t} = (H_{t+1,t} - L_{t+1,t-1} L_{t,t-1}^T) L_tt^-T
//   L_{t+2,t} = H_{t+2,t} L_tt^-T
// followed by block forward / backward substitution: O(T nv^3) instead of O((T nv)^3).
//
// Precision: the normal matrix has condition ~1e8 (acceleration stiffness
// (w/dt^2)^2 against a 1e-6 regularisation).  A float32 factorization fails there,
// and even float32 Jacobian entries (relative error ~1e-7) move the Gauss-Newton
// step by ~1e-1 rad along the weakly constrained directions, so the whole
// trajectory solver — iterate, residuals, pose Jacobians, bands, factorization,
// solves — is float64.
//
// After the solve, the gradient of the final cost w.r.t. the goal pose (a right
// perturbation T_goal exp(eps)) is the adjoint -w_goal^2 Jl^-1(xi)^T xi of the
// goal term (envelope theorem: the other terms do not depend on the target and
// dcost/dx = 0 at the optimum); Jl^-1(xi) = Jr^-1(-xi), exact 20-term series.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/br_b200.h"
#include "br_common.cuh"
#include "br_fk.cuh"
#include "br_lie.cuh"

namespace br {

struct TrajParams {
  br_tree_t tree;
  br_traj_settings_t s;
  int32_t frame_id, T;
  int64_t n;
  const float* x0;
  const float* xref;
  const float* goal;
  const float* start;
  float* x;
  int32_t* iters;
  int32_t* status;
  float* cost;
  float* goal_grad;
};

struct TrajLayout {
  // doubles
  int x, xn, xref, g, delta, D, E1, E2, dinvt, Jg, Js, rg, rs, jtjg, jtjs, pA, pB;
  int total_doubles;
  // ints / floats (in units of doubles)
  int parent, jtype, idxq, cjoint, ckind, axis, place, caxis, anc, lower, upper, misc;
  int total;
  __host__ __device__ TrajLayout(int nj, int nq, int nv, int T) {
    int o = 0;
    auto take = [&](int n) { int r = o; o += (n + 1) & ~1; return r; };  // 16-byte aligned
    x = take(T * nv); xn = take(T * nv); xref = take(T * nv); g = take(T * nv); delta = take(T * nv);
    D = take(T * nv * nv); E1 = take(T * nv * nv); E2 = take(T * nv * nv); dinvt = take(T * nv);
    Jg = take(6 * nv); Js = take(6 * nv); rg = take(8); rs = take(8); jtjg = take(nv * nv); jtjs = take(nv * nv);
    pA = take(8 * nj); pB = take(8 * nj);
    total_doubles = o;
    // 4-byte arrays: count in doubles (2 per double)
    auto take4 = [&](int n) { int r = o; o += ((n + 3) & ~3) / 2; return r; };
    parent = take4(nj); jtype = take4(nj); idxq = take4(nj); cjoint = take4(nv); ckind = take4(nv);
    axis = take4(4 * nj); place = take4(8 * nj); caxis = take4(4 * nv); anc = take4(2 * nj);
    lower = take4(nq); upper = take4(nq); misc = take4(8);
    total = o;
  }
};

__device__ __forceinline__ DPose ldd8(const double* p) {
  return DPose{d3(p[0], p[1], p[2]), make_double4(p[4], p[5], p[6], p[7])};
}
__device__ __forceinline__ void std8d(double* p, const DPose& P) {
  p[0] = P.t.x; p[1] = P.t.y; p[2] = P.t.z; p[3] = 0.0;
  p[4] = P.q.x; p[5] = P.q.y; p[6] = P.q.z; p[7] = P.q.w;
}

__global__ void traj_gn_kernel(const TrajParams P) {
  extern __shared__ __align__(16) double sm[];
  const br_tree_t& tree = P.tree;
  const int nj = tree.njoints, nq = tree.nq, nv = tree.nv, T = P.T, lane = threadIdx.x;
  const int64_t traj = blockIdx.x;
  if (traj >= P.n) return;
  const TrajLayout L(nj, nq, nv, T);
  double* x = sm + L.x;
  double* xn = sm + L.xn;
  double* xref = sm + L.xref;
  double* g = sm + L.g;
  double* delta = sm + L.delta;
  double* D = sm + L.D;
  double* E1 = sm + L.E1;
  double* E2 = sm + L.E2;
  double* dinvt = sm + L.dinvt;  // 1 / L_tt[k][k] of every diagonal block
  double* Jg = sm + L.Jg;
  double* Js = sm + L.Js;
  double* rg = sm + L.rg;
  double* rs = sm + L.rs;
  double* jtjg = sm + L.jtjg;
  double* jtjs = sm + L.jtjs;
  double* pA = sm + L.pA;
  double* pB = sm + L.pB;
  int* parent = reinterpret_cast<int*>(sm + L.parent);
  int* jtype = reinterpret_cast<int*>(sm + L.jtype);
  int* idxq = reinterpret_cast<int*>(sm + L.idxq);
  int* cjoint = reinterpret_cast<int*>(sm + L.cjoint);
  int* ckind = reinterpret_cast<int*>(sm + L.ckind);
  float* axis = reinterpret_cast<float*>(sm + L.axis);
  float* place = reinterpret_cast<float*>(sm + L.place);
  float* caxis = reinterpret_cast<float*>(sm + L.caxis);
  int* ancA = reinterpret_cast<int*>(sm + L.anc);
  int* ancB = ancA + nj;
  float* lower = reinterpret_cast<float*>(sm + L.lower);
  float* upper = reinterpret_cast<float*>(sm + L.upper);
  const br_traj_settings_t& S = P.s;
  const double c = (double)S.w_accel / ((double)S.dt * (double)S.dt);
  const double c2 = c * c;
  const double wl = S.w_limit, wr = S.w_ref, wg = S.w_goal, ws = S.w_start;
  const bool has_start = P.start != nullptr && S.w_start > 0.f;
  const bool has_goal = S.w_goal > 0.f;
  const int n = T * nv;

  for (int j = lane; j < nj; j += kWarp) {
    parent[j] = tree.parent[j];
    jtype[j] = tree.jtype[j];
    idxq[j] = tree.idx_q[j];
    for (int k = 0; k < 4; ++k) axis[4 * j + k] = tree.axis[4 * j + k];
    for (int k = 0; k < 8; ++k) place[8 * j + k] = tree.placement[8 * j + k];
  }
  for (int k = lane; k < nv; k += kWarp) {
    cjoint[k] = tree.col_joint[k];
    ckind[k] = tree.col_kind[k];
    for (int m = 0; m < 4; ++m) caxis[4 * k + m] = tree.col_axis[4 * k + m];
  }
  for (int i = lane; i < nq; i += kWarp) {
    lower[i] = tree.lower[i];
    upper[i] = tree.upper[i];
  }
  const float* x0 = P.x0 + traj * (int64_t)n;
  const float* xr = (P.xref ? P.xref : P.x0) + traj * (int64_t)n;
  for (int i = lane; i < n; i += kWarp) {
    x[i] = x0[i];
    xref[i] = xr[i];
  }
  const int fpar = tree.frame_parent[P.frame_id];
  const Pose fpl = load_pose8(tree.frame_placement + 8 * P.frame_id);
  const unsigned long long sup = tree.support[fpar];
  Pose tgt_goal, tgt_start;
  {
    const float* tp = P.goal + traj * 7;
    tgt_goal = Pose{f3(tp[0], tp[1], tp[2]), make_float4(tp[3], tp[4], tp[5], tp[6])};
    if (has_start) {
      const float* sp = P.start + traj * 7;
      tgt_start = Pose{f3(sp[0], sp[1], sp[2]), make_float4(sp[3], sp[4], sp[5], sp[6])};
    }
  }
  __syncwarp();

  // float64 FK of knot t of trajectory `xs`; returns the world pose buffer
  auto fk = [&](const double* xs, int t) -> double* {
    const double* q = xs + t * nv;
    for (int j = lane; j < nj; j += kWarp) {
      const Pose Pj = load_pose8(place + 8 * j);
      const DPose Lj = dlocal_transform(jtype[j], DPose{d3(Pj.t.x, Pj.t.y, Pj.t.z),
                                                        make_double4(Pj.q.x, Pj.q.y, Pj.q.z, Pj.q.w)},
                                        axis + 4 * j, q + idxq[j]);
      std8d(pA + 8 * j, Lj);
      ancA[j] = parent[j];
    }
    __syncwarp();
    double* A = pA;
    double* B = pB;
    int* aA = ancA;
    int* aB = ancB;
    for (int r = 0; r < tree.rounds; ++r) {
      for (int j = lane; j < nj; j += kWarp) {
        const int a = aA[j];
        if (a >= 0) {
          std8d(B + 8 * j, dcompose(ldd8(A + 8 * a), ldd8(A + 8 * j)));
          aB[j] = aA[a];
        } else {
          std8d(B + 8 * j, ldd8(A + 8 * j));
          aB[j] = -1;
        }
      }
      __syncwarp();
      double* tp = A; A = B; B = tp;
      int* ta = aA; aA = aB; aB = ta;
    }
    return A;
  };
  // pose term at knot t: xi (double, into r[0..5]); if J != null also J = Jr^-1 blockdiag(R^T,R^T) J_lwa (6 x nv)
  auto pose_term = [&](const double* xs, int t, const Pose& target, double* r, double* J) {
    double* pose = fk(xs, t);
    const DPose Tee = dcompose(ldd8(pose + 8 * fpar),
                               DPose{d3(fpl.t.x, fpl.t.y, fpl.t.z), make_double4(fpl.q.x, fpl.q.y, fpl.q.z, fpl.q.w)});
    double3 v, w;
    dse3_log(dcompose(dinverse(DPose{d3(target.t.x, target.t.y, target.t.z),
                                     make_double4(target.q.x, target.q.y, target.q.z, target.q.w)}), Tee), v, w);
    if (lane == 0) { r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = w.x; r[4] = w.y; r[5] = w.z; }
    if (J) {
      const DJrInv Jr = djr_inv_se3<9>(v, w);
      const double4 qc = dqconj(Tee.q);
      for (int k = lane; k < nv; k += kWarp) {
        double3 ol = d3(0, 0, 0), oa = d3(0, 0, 0);
        if ((sup >> cjoint[k]) & 1ull) {
          const DPose Tj = ldd8(pose + 8 * cjoint[k]);
          const double3 a = dqrot(Tj.q, d3(caxis[4 * k], caxis[4 * k + 1], caxis[4 * k + 2]));
          double3 lin, ang;
          if (ckind[k] == 0) {
            lin = dcross(a, dsub(Tee.t, Tj.t));
            ang = a;
          } else {
            lin = a;
            ang = d3(0, 0, 0);
          }
          djr_inv_apply(Jr, dqrot(qc, lin), dqrot(qc, ang), ol, oa);
        }
        J[0 * nv + k] = ol.x; J[1 * nv + k] = ol.y; J[2 * nv + k] = ol.z;
        J[3 * nv + k] = oa.x; J[4 * nv + k] = oa.y; J[5 * nv + k] = oa.z;
      }
    }
    __syncwarp();
  };
  auto warp_sum = [&](double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  };
  // total cost 0.5 |r|^2 at xs (pose terms evaluated into rg / rs)
  auto cost_of = [&](const double* xs) -> double {
    double acc = 0.0;
    if (has_goal) pose_term(xs, T - 1, tgt_goal, rg, nullptr);
    if (has_start) pose_term(xs, 0, tgt_start, rs, nullptr);
    for (int e = lane; e < (T - 2) * nv; e += kWarp) {
      const double a = c * (xs[e + 2 * nv] - 2.0 * xs[e + nv] + xs[e]);
      acc += a * a;
    }
    for (int e = lane; e < n; e += kWarp) {
      const int i = e % nv;
      const double lo = fmax((double)lower[i] - xs[e], 0.0), hi = fmax(xs[e] - (double)upper[i], 0.0);
      const double d = xs[e] - xref[e];
      acc += wl * wl * (lo * lo + hi * hi) + wr * wr * d * d;
    }
    acc = warp_sum(acc);
    double pc = 0.0;
    for (int k = 0; k < 6; ++k) {
      if (has_goal) pc += wg * wg * rg[k] * rg[k];
      if (has_start) pc += ws * ws * rs[k] * rs[k];
    }
    __syncwarp();
    return 0.5 * (acc + pc);
  };
  // J^T J of the pose terms and g = J^T r at x; returns |g|
  auto build = [&]() -> double {
    if (has_goal) pose_term(x, T - 1, tgt_goal, rg, Jg);
    if (has_start) pose_term(x, 0, tgt_start, rs, Js);
    for (int e = lane; e < nv * nv; e += kWarp) {
      const int i = e / nv, j = e - i * nv;
      double a = 0.0, b = 0.0;
      for (int r = 0; r < 6; ++r) {
        if (has_goal) a += Jg[r * nv + i] * Jg[r * nv + j];
        if (has_start) b += Js[r * nv + i] * Js[r * nv + j];
      }
      jtjg[e] = wg * wg * a;
      jtjs[e] = ws * ws * b;
    }
    double gg = 0.0;
    for (int e = lane; e < n; e += kWarp) {
      const int t = e / nv, i = e - t * nv;
      double acc = 0.0;
      // acceleration rows s = t, t-1, t-2 with coefficients +1, -2, +1 at knot t
      auto arow = [&](int s) { return c * (x[(s + 2) * nv + i] - 2.0 * x[(s + 1) * nv + i] + x[s * nv + i]); };
      if (t <= T - 3) acc += c * arow(t);
      if (t - 1 >= 0 && t - 1 <= T - 3) acc += -2.0 * c * arow(t - 1);
      if (t - 2 >= 0) acc += c * arow(t - 2);
      if (x[e] < (double)lower[i]) acc -= wl * wl * ((double)lower[i] - x[e]);
      if (x[e] > (double)upper[i]) acc += wl * wl * (x[e] - (double)upper[i]);
      acc += wr * wr * (x[e] - xref[e]);
      if (has_goal && t == T - 1)
        for (int r = 0; r < 6; ++r) acc += wg * wg * Jg[r * nv + i] * rg[r];
      if (has_start && t == 0)
        for (int r = 0; r < 6; ++r) acc += ws * ws * Js[r * nv + i] * rs[r];
      g[e] = acc;
      gg += acc * acc;
    }
    gg = warp_sum(gg);
    __syncwarp();
    return sqrt(gg);
  };
  // assemble the bands of J^T J + damp I at x
  auto assemble = [&](double damp) {
    for (int e = lane; e < T * nv * nv; e += kWarp) {
      const int t = e / (nv * nv), ij = e - t * nv * nv, i = ij / nv, j = ij - i * nv;
      double d = 0.0, e1 = 0.0, e2 = 0.0;
      if (i == j) {
        // diagonal: acceleration coefficient squares at knot t
        double a = 0.0;
        if (t <= T - 3) a += 1.0;
        if (t - 1 >= 0 && t - 1 <= T - 3) a += 4.0;
        if (t - 2 >= 0) a += 1.0;
        const double xv = x[t * nv + i];
        d = c2 * a + wr * wr + damp;
        if (xv < (double)lower[i]) d += wl * wl;
        if (xv > (double)upper[i]) d += wl * wl;
        double b = 0.0;                       // block (t+1, t)
        if (t <= T - 3) b += -2.0;
        if (t - 1 >= 0 && t <= T - 2) b += -2.0;
        e1 = (t <= T - 2) ? c2 * b : 0.0;
        e2 = (t <= T - 3) ? c2 : 0.0;        // block (t+2, t)
      }
      if (has_goal && t == T - 1) d += jtjg[ij];
      if (has_start && t == 0) d += jtjs[ij];
      D[e] = d;
      E1[e] = e1;
      E2[e] = e2;
    }
    __syncwarp();
  };
  // C -= A B^T (nv x nv blocks)
  auto sub_abt = [&](double* C, const double* A, const double* B) {
    for (int e = lane; e < nv * nv; e += kWarp) {
      const int i = e / nv, j = e - i * nv;
      double acc = C[e];
      for (int k = 0; k < nv; ++k) acc -= A[i * nv + k] * B[j * nv + k];
      C[e] = acc;
    }
    __syncwarp();
  };
  // bandwidth-2 block Cholesky in place; solve L L^T delta = -g
  auto factor_solve = [&]() -> bool {
    const int b2 = nv * nv;
    for (int t = 0; t < T; ++t) {
      double* Dt = D + t * b2;
      if (t >= 1) sub_abt(Dt, E1 + (t - 1) * b2, E1 + (t - 1) * b2);
      if (t >= 2) sub_abt(Dt, E2 + (t - 2) * b2, E2 + (t - 2) * b2);
      if (t >= 1 && t + 1 < T) sub_abt(E1 + t * b2, E2 + (t - 1) * b2, E1 + (t - 1) * b2);
      for (int k = 0; k < nv; ++k) {                               // chol(D_t)
        const double dkk = Dt[k * nv + k];
        if (!(dkk > 0.0)) return false;
        const double s = sqrt(dkk);
        const double inv = 1.0 / s;                                // every lane: no broadcast needed
        __syncwarp();
        if (lane > k && lane < nv) Dt[lane * nv + k] *= inv;
        if (lane == k) { Dt[k * nv + k] = s; dinvt[t * nv + k] = inv; }
        __syncwarp();
        for (int e = lane; e < b2; e += kWarp) {
          const int i = e / nv, j = e - i * nv;
          if (j > k && i >= j) Dt[e] -= Dt[i * nv + k] * Dt[j * nv + k];
        }
        __syncwarp();
      }
      // off-diagonal blocks: X <- X L_tt^-T, lanes 0..nv-1 rows of E1_t, lanes 16.. rows of E2_t
      double* X = nullptr;
      int row = -1;
      if (lane < nv && t + 1 < T) { X = E1 + t * b2; row = lane; }
      if (lane >= 16 && lane - 16 < nv && t + 2 < T) { X = E2 + t * b2; row = lane - 16; }
      if (X) {
        double* xr = X + row * nv;
        const double* di = dinvt + t * nv;
        for (int j = 0; j < nv; ++j) {
          double v = xr[j];
          for (int k = 0; k < j; ++k) v -= xr[k] * Dt[j * nv + k];
          xr[j] = v * di[j];
        }
      }
      __syncwarp();
    }
    // forward: L y = -g (y in delta).  Lane i < nv owns row i of each knot; the 7x7
    // diagonal solve broadcasts one finished entry per step by shuffle.
    const double* Ld = D;
    for (int t = 0; t < T; ++t) {
      double v = 0.0;
      if (lane < nv) {
        v = -g[t * nv + lane];
        if (t >= 1) for (int k = 0; k < nv; ++k) v -= E1[(t - 1) * b2 + lane * nv + k] * delta[(t - 1) * nv + k];
        if (t >= 2) for (int k = 0; k < nv; ++k) v -= E2[(t - 2) * b2 + lane * nv + k] * delta[(t - 2) * nv + k];
      }
      const double* Lt = Ld + t * b2;
      const double* di = dinvt + t * nv;
      for (int j = 0; j < nv; ++j) {
        const double yj = __shfl_sync(0xffffffffu, v, j) * di[j];
        if (lane == j) v = yj;
        else if (lane > j && lane < nv) v -= Lt[lane * nv + j] * yj;
      }
      if (lane < nv) delta[t * nv + lane] = v;
      __syncwarp();
    }
    // backward: L^T dx = y
    for (int t = T - 1; t >= 0; --t) {
      double v = 0.0;
      if (lane < nv) {
        v = delta[t * nv + lane];
        if (t + 1 < T) for (int k = 0; k < nv; ++k) v -= E1[t * b2 + k * nv + lane] * delta[(t + 1) * nv + k];
        if (t + 2 < T) for (int k = 0; k < nv; ++k) v -= E2[t * b2 + k * nv + lane] * delta[(t + 2) * nv + k];
      }
      const double* Lt = Ld + t * b2;
      const double* di = dinvt + t * nv;
      for (int j = nv - 1; j >= 0; --j) {
        const double xj = __shfl_sync(0xffffffffu, v, j) * di[j];
        if (lane == j) v = xj;
        else if (lane < j) v -= Lt[j * nv + lane] * xj;
      }
      __syncwarp();
      if (lane < nv) delta[t * nv + lane] = v;
      __syncwarp();
    }
    return true;
  };

  // ---- GN / LM loop (gauss_newton.py:27-76, levenberg_marquardt.py:83-135) ----
  const bool lm = S.optimizer == BR_OPT_LM;
  double cost = cost_of(x);
  double lam = lm ? (double)S.lam0 : 0.0;
  double gnorm = 0.0;
  bool need = true;
  int status = BR_IK_MAXITER, flags = 0, it = 0;
  for (; it < S.max_iter; ++it) {
    if (need) { gnorm = build(); need = false; }
    assemble(lm ? lam : (double)S.gn_eps);
    if (!factor_solve()) {
      flags |= BR_IK_FLAG_REGULARIZED;
      bool ok = false;
      double extra = 1e-9;
      for (int k = 0; k < 8 && !ok; ++k, extra *= 10.0) {
        assemble((lm ? lam : (double)S.gn_eps) + extra);
        ok = factor_solve();
      }
      if (!ok) {
        for (int e = lane; e < n; e += kWarp) delta[e] = 0.0;
        __syncwarp();
      }
    }
    for (int e = lane; e < n; e += kWarp) xn[e] = x[e] + delta[e];  // knot retraction: q + dv (nq == nv)
    __syncwarp();
    const double cn = cost_of(xn);
    if (!isfinite(cn)) flags |= BR_IK_FLAG_NONFINITE;
    bool accept = !lm || cn < cost;
    if (accept) {
      for (int e = lane; e < n; e += kWarp) x[e] = xn[e];
      __syncwarp();
      cost = cn;
      need = true;
      if (lm) lam = fmax(lam / S.factor, (double)S.lam_min);
      if (gnorm < S.tol) { status = BR_IK_CONVERGED; ++it; break; }
    } else {
      lam = fmin(lam * S.factor, (double)S.lam_max);
    }
  }
  float* xo = P.x + traj * (int64_t)n;
  for (int e = lane; e < n; e += kWarp) xo[e] = (float)x[e];
  if (P.goal_grad && has_goal) {
    pose_term(x, T - 1, tgt_goal, rg, nullptr);
    if (lane == 0) {
      const double3 v = d3(rg[0], rg[1], rg[2]);
      const double3 w = d3(rg[3], rg[4], rg[5]);
      const DJrInv Jl = djr_inv_se3<20>(dscale(v, -1.0), dscale(w, -1.0));   // Jl^-1(xi) = Jr^-1(-xi)
      double3 gl, ga;
      djr_inv_T_apply(Jl, v, w, gl, ga);
      const double k = -wg * wg;
      float* o = P.goal_grad + traj * 6;
      o[0] = (float)(k * gl.x); o[1] = (float)(k * gl.y); o[2] = (float)(k * gl.z);
      o[3] = (float)(k * ga.x); o[4] = (float)(k * ga.y); o[5] = (float)(k * ga.z);
    }
  }
  if (lane == 0) {
    P.iters[traj] = it;
    P.status[traj] = status | (flags << 8);
    P.cost[traj] = (float)cost;
  }
}

}  // namespace br

using namespace br;

extern "C" int br_trajopt_solve(const br_tree_t* tree, int32_t frame_id, int64_t n_traj, int32_t knots,
                                const float* x0, const float* x_ref, const float* goal, const float* start,
                                const br_traj_settings_t* settings, float* x, int32_t* iters, int32_t* status,
                                float* cost, float* goal_grad, void* stream) {
  int st = validate_tree(tree);
  if (st) return st;
  if (!settings || n_traj < 0 || knots < 3) return BR_EINVAL;
  if (knots > BR_MAX_TRAJ_KNOTS || tree->nv > BR_MAX_TRAJ_NV) return BR_ETOOBIG;
  if (tree->nq != tree->nv) return BR_EINVAL;  // fixed-base trees: difference(q0, q1) = q1 - q0
  {
    const int ok = (1 << BR_JOINT_FIXED) | (1 << BR_JOINT_REVOLUTE) | (1 << BR_JOINT_PRISMATIC) |
                   (1 << BR_JOINT_TRANSLATION);
    if (tree->kinds == 0 || (tree->kinds & ~ok)) return BR_EINVAL;  // q + v kinds only
  }
  if (frame_id < 0 || frame_id >= tree->nframes) return BR_EINVAL;
  if (n_traj == 0) return BR_OK;
  if (!x0 || !goal || !x || !iters || !status || !cost) return BR_EINVAL;
  if (settings->max_iter < 0 || !(settings->dt > 0.f)) return BR_EINVAL;
  TrajParams p = {};
  p.tree = *tree;
  p.s = *settings;
  p.frame_id = frame_id;
  p.T = knots;
  p.n = n_traj;
  p.x0 = x0; p.xref = x_ref; p.goal = goal; p.start = start;
  p.x = x; p.iters = iters; p.status = status; p.cost = cost; p.goal_grad = goal_grad;
  const TrajLayout L(tree->njoints, tree->nq, tree->nv, knots);
  const size_t bytes = (size_t)L.total * sizeof(double);
  const DeviceInfo& dev = device_info();
  if ((int64_t)bytes > dev.max_smem_optin) return BR_ETOOBIG;
  static int configured[16] = {0};
  if ((int)bytes > configured[dev.device & 15]) {
    cudaError_t e = cudaFuncSetAttribute(traj_gn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    configured[dev.device & 15] = (int)bytes;
  }
  if (n_traj > 0x7fffffff) return BR_ETOOBIG;
  traj_gn_kernel<<<(unsigned)n_traj, kWarp, bytes, (cudaStream_t)stream>>>(p);
  return (int)cudaGetLastError();
}

// traj_gn.cu — batched trajectory optimisation (Gauss-Newton / LM), one warp per
// trajectory, Newton step in nested-dissection order.
//
// Reference: solve_trajopt with knot parameterisation
// (src/better_robot/tasks/trajopt.py:84-230) flattens a (T, nq) trajectory into one
// least-squares problem and solves the dense (T*nv)^2 normal equations with a
// dense Cholesky every iteration (448 x 448 for T = 64, nv = 7).  The stack here is
//   goal  : PoseResidual at knot T-1        (TimeIndexedResidual, residuals/temporal.py:20-126)
//   start : PoseResidual at knot 0          (optional)
//   accel : (d_{s+1} - d_s)/dt^2, d_t = difference(q_t, q_{t+1}) (= q_{t+1} - q_t for q + v
//           joints)                         (AccelerationResidual, residuals/smoothness.py:98-161)
//   limits: JointPositionLimit at every knot (residuals/limits.py:56-86)
//   ref   : difference(q_ref_t, q_t)        (ReferenceTrajectoryResidual, residuals/regularization.py:133-152)
// each with a CostStack item weight.  In its J^T J + damp I every term except the
// two pose terms acts on one DOF at a time: the acceleration rows couple knots
// t, t+1, t+2 of the same DOF, limits / reference / damping are diagonal.  So H is
// nv independent scalar PENTA-diagonal T x T matrices (one per DOF) plus the dense
// nv x nv pose blocks at knots 0 and T-1.  The kernel solves it in nested-dissection
// order: the interior knots 1..T-2 of each DOF first — lane i runs the banded
// LDL^T of DOF i and three solves (right-hand side and the two columns that tie the
// interior to knots 0 and T-1) — leaving a 2nv x 2nv Schur complement on the
// boundary knots,
//   S = H_bb - H_bI P^-1 H_Ib,   P = blockdiag_i(P_i) the per-DOF interior bands,
// which the warp factors with a dense Cholesky; the interior step follows by one
// update.  This is the exact Cholesky of a symmetric permutation of H (no
// approximation): O(T nv) sequential work per iteration instead of the O(T nv^3) of
// a block-banded factorization or the O((T nv)^3) of the dense one.
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
  int x, xn, dd, dr, g, delta, bl1, bdi, Sb, sdi, rb, zb, Jg, Js, rg, rs, jtjg, jtjs, pA, pB, red;
  int total_doubles;
  // 4-byte arrays (offsets in doubles)
  int xref, parent, jtype, idxq, idxv, dofq, cjoint, ckind, axis, place, caxis, anc, lower, upper;
  int total;
  __host__ __device__ TrajLayout(int nj, int nq, int nv, int T, bool floating) {
    int o = 0;
    auto take = [&](int n) { int r = o; o += (n + 1) & ~1; return r; };  // 16-byte aligned
    const int nb = 2 * nv;
    x = take(T * nq); xn = take(T * nq); g = take(T * nv); delta = take(T * nv);
    // knot differences difference(x_t, x_{t+1}) and difference(xref_t, x_t) of the last
    // evaluated trajectory (kManifold variant; the other subtracts inline)
    dd = take(floating ? T * nv : 0); dr = take(floating ? T * nv : 0);
    // per-DOF interior band factors (index p * nv + i, p = knot - 1): L[p][p-1] and 1 / D[p]
    // (L[p][p-2] = c^2 / D[p-2] is rebuilt from 1 / D)
    bl1 = take(T * nv); bdi = take(T * nv);
    Sb = take(nb * (nb + 1) / 2); sdi = take(nb); rb = take(nb); zb = take(nb);  // boundary Schur complement
    Jg = take(6 * nv); Js = take(6 * nv); rg = take(8); rs = take(8);
    jtjg = take(nv * (nv + 1) / 2); jtjs = take(nv * (nv + 1) / 2);              // packed lower
    pA = take(16 * nj); pB = take(16 * nj);   // FK buffers of the two pose terms (goal, start)
    red = take(32);                           // per-warp partial sums of the block reductions
    total_doubles = o;
    auto take4 = [&](int n) { int r = o; o += ((n + 3) & ~3) / 2; return r; };
    xref = take4(T * nq);                     // float32, as given
    parent = take4(nj); jtype = take4(nj); idxq = take4(nj); idxv = take4(nj); dofq = take4(nv);
    cjoint = take4(nv); ckind = take4(nv);
    axis = take4(4 * nj); place = take4(8 * nj); caxis = take4(4 * nv); anc = take4(8 * nj);
    lower = take4(nq); upper = take4(nq);
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

// 1 / d for d > 0 (a pivot): the hardware reciprocal estimate refined by two Newton steps
// r <- r + r (1 - d r), each of which squares the relative error (~2^-23 -> 2^-46 -> below
// double rounding); within an ulp or two of 1.0 / d at a fraction of the division's latency.
__device__ __forceinline__ double fast_rcp(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}
// 1 / sqrt(x) for x > 0: estimate + two Newton steps y <- y (3 - x y^2) / 2
__device__ __forceinline__ double fast_rsqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = y * fma(-0.5 * x * y, y, 1.5);
  return y * fma(-0.5 * x * y, y, 1.5);
}

// packed lower-triangle index p -> (a, b), b <= a, p = a (a + 1) / 2 + b: approximate square
// root, made exact by its two integer corrections
__device__ __forceinline__ int2 tri_decode(int p) {
  int a = (int)((sqrtf(8.f * p + 1.f) - 1.f) * 0.5f);
  if ((a + 1) * (a + 2) / 2 <= p) ++a;
  if (a * (a + 1) / 2 > p) --a;
  return make_int2(a, p - a * (a + 1) / 2);
}
__device__ __forceinline__ int tri_at(int r, int c) { return r * (r + 1) / 2 + c; }  // r >= c

// Threads per trajectory: the per-DOF interior chains take one thread each (nv <= 64),
// the two pose terms one warp each, everything else strides over the block.
constexpr int kTrajThreads = 128;

// kManifold: the tree has joints whose configuration is not their tangent coordinates
// (free-flyer, spherical, planar, unbounded revolute): knot differences and the retraction go
// through Model.difference / Model.integrate; otherwise they are q1 - q0 and q + v.
template <bool kManifold>
__global__ void __launch_bounds__(kTrajThreads) traj_gn_kernel(const TrajParams P) {
  extern __shared__ __align__(16) double sm[];
  const br_tree_t& tree = P.tree;
  const int nj = tree.njoints, nq = tree.nq, nv = tree.nv, T = P.T;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NT = kTrajThreads, NW = kTrajThreads / kWarp;
  const int64_t traj = blockIdx.x;
  if (traj >= P.n) return;
  const TrajLayout L(nj, nq, nv, T, kManifold);
  double* x = sm + L.x;
  double* xn = sm + L.xn;
  double* g = sm + L.g;
  double* delta = sm + L.delta;
  double* bl1 = sm + L.bl1;
  double* bdi = sm + L.bdi;
  double* Sb = sm + L.Sb;
  double* sdi = sm + L.sdi;
  double* rb = sm + L.rb;
  double* zb = sm + L.zb;
  double* Jg = sm + L.Jg;
  double* Js = sm + L.Js;
  double* rg = sm + L.rg;
  double* rs = sm + L.rs;
  double* jtjg = sm + L.jtjg;
  double* jtjs = sm + L.jtjs;
  double* pA = sm + L.pA;
  double* pB = sm + L.pB;
  double* red = sm + L.red;
  float* xref = reinterpret_cast<float*>(sm + L.xref);
  int* parent = reinterpret_cast<int*>(sm + L.parent);
  int* jtype = reinterpret_cast<int*>(sm + L.jtype);
  int* idxq = reinterpret_cast<int*>(sm + L.idxq);
  int* idxv = reinterpret_cast<int*>(sm + L.idxv);
  int* dofq = reinterpret_cast<int*>(sm + L.dofq);  // q slot of a DOF with a position limit, else -1
  double* dd = sm + L.dd;
  double* dr = sm + L.dr;
  int* cjoint = reinterpret_cast<int*>(sm + L.cjoint);
  int* ckind = reinterpret_cast<int*>(sm + L.ckind);
  float* axis = reinterpret_cast<float*>(sm + L.axis);
  float* place = reinterpret_cast<float*>(sm + L.place);
  float* caxis = reinterpret_cast<float*>(sm + L.caxis);
  int* ancA = reinterpret_cast<int*>(sm + L.anc);
  int* ancB = ancA + 2 * nj;
  float* lower = reinterpret_cast<float*>(sm + L.lower);
  float* upper = reinterpret_cast<float*>(sm + L.upper);
  const br_traj_settings_t& S = P.s;
  const double c = (double)S.w_accel / ((double)S.dt * (double)S.dt);
  const double c2 = c * c;
  const double wl = S.w_limit, wr = S.w_ref, wg = S.w_goal, ws = S.w_start;
  const bool has_start = P.start != nullptr && S.w_start > 0.f;
  const bool has_goal = S.w_goal > 0.f;
  const int n = T * nv, nqT = T * nq, nb = 2 * nv;
  const FastDiv divj(nj > 0 ? nj : 1), divv(nv > 0 ? nv : 1), divq(nq > 0 ? nq : 1);

  for (int j = tid; j < nj; j += NT) {
    parent[j] = tree.parent[j];
    jtype[j] = tree.jtype[j];
    idxq[j] = tree.idx_q[j];
    idxv[j] = tree.idx_v[j];
    for (int k = 0; k < 4; ++k) axis[4 * j + k] = tree.axis[4 * j + k];
    for (int k = 0; k < 8; ++k) place[8 * j + k] = tree.placement[8 * j + k];
  }
  for (int k = tid; k < nv; k += NT) {
    cjoint[k] = tree.col_joint[k];
    ckind[k] = tree.col_kind[k];
    for (int m = 0; m < 4; ++m) caxis[4 * k + m] = tree.col_axis[4 * k + m];
  }
  for (int i = tid; i < nq; i += NT) {
    lower[i] = tree.lower[i];
    upper[i] = tree.upper[i];
  }
  __syncthreads();
  for (int j = tid; j < nj; j += NT) {              // limits.py:36-48: nq == nv joints only
    const int jt = jtype[j];
    const bool vec = joint_is_vector(jt);
    for (int k = 0; k < joint_nv(jt); ++k) dofq[idxv[j] + k] = vec ? idxq[j] + k : -1;
  }
  const float* x0 = P.x0 + traj * (int64_t)nqT;
  const float* xr = (P.xref ? P.xref : P.x0) + traj * (int64_t)nqT;
  for (int i = tid; i < nqT; i += NT) {
    x[i] = x0[i];
    xref[i] = xr[i];
  }
  const int fpar = tree.frame_parent[P.frame_id];
  const Pose fpl = load_pose8(tree.frame_placement + 8 * P.frame_id);
  const unsigned long long sup = tree.support[fpar];
  __syncthreads();

  auto warp_sum = [&](double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  };
  // sum over the block; every thread gets the same value (the warps' partials are added in
  // warp order by every thread)
  auto block_sum = [&](double v) -> double {
    v = warp_sum(v);
    __syncthreads();                                  // the previous reduction's reads are done
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += red[w];
    return s;
  };
  // float64 FK of knot t of trajectory `xs` by one warp (pose term h: buffers pA / pB + 8 nj h,
  // ancA / ancB + nj h); returns the world poses
  auto fk = [&](const double* xs, int t, int h) -> double* {
    const double* q = xs + t * nq;
    double* A = pA + 8 * nj * h;
    double* B = pB + 8 * nj * h;
    int* aA = ancA + nj * h;
    int* aB = ancB + nj * h;
    for (int j = lane; j < nj; j += kWarp) {
      const Pose Pj = load_pose8(place + 8 * j);
      const DPose Lj = dlocal_transform(jtype[j], DPose{d3(Pj.t.x, Pj.t.y, Pj.t.z),
                                                        make_double4(Pj.q.x, Pj.q.y, Pj.q.z, Pj.q.w)},
                                        axis + 4 * j, q + idxq[j]);
      std8d(A + 8 * j, Lj);
      aA[j] = parent[j];
    }
    __syncwarp();
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
  // both pose terms at xs, warp 0 the goal (knot T-1), warp 1 the start (knot 0): xi (into
  // rg / rs); with want_J also J = Jr^-1 blockdiag(R^T,R^T) J_lwa (6 x nv, into Jg / Js).
  // A term that is not in the problem (weight 0 or no start pose) is skipped.  With `reuse`
  // the knot's FK and xi are those the last call left (the build follows the cost evaluation
  // of the same point, and nothing in between writes the pose buffers).
  auto pose_terms = [&](const double* xs, bool want_J, bool reuse) __attribute__((always_inline)) {
    if (warp < 2) {
      const int h = warp;
      const bool active = h == 0 ? has_goal : has_start;
      if (active) {
        const float* tp = (h == 0 ? P.goal : P.start) + traj * 7;   // the term's target pose
        const DPose target{d3(tp[0], tp[1], tp[2]), make_double4(tp[3], tp[4], tp[5], tp[6])};
        double* r = h == 0 ? rg : rs;
        double* J = h == 0 ? Jg : Js;
        double* pose = reuse ? ((tree.rounds & 1) ? pB : pA) + 8 * nj * h : fk(xs, h == 0 ? T - 1 : 0, h);
        const DPose Tee = dcompose(ldd8(pose + 8 * fpar), DPose{d3(fpl.t.x, fpl.t.y, fpl.t.z),
                                                                make_double4(fpl.q.x, fpl.q.y, fpl.q.z, fpl.q.w)});
        double3 v, w;
        if (reuse) {
          v = d3(r[0], r[1], r[2]);
          w = d3(r[3], r[4], r[5]);
        } else {
          dse3_log(dcompose(dinverse(target), Tee), v, w);
          if (lane == 0) { r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = w.x; r[4] = w.y; r[5] = w.z; }
        }
        if (want_J) {
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
      }
    }
    // the build reads J next; a cost evaluation reads xi only after its block sum's barriers
    if (want_J) __syncthreads();
  };
  // dd[t] = difference(xs_t, xs_{t+1}) (t < T-1) and dr[t] = difference(xref_t, xs_t)
  // (model.py:176-190): free-flyer log(q_a^-1 q_b) (free_flyer.py:53-57), spherical
  // log(normalize(q_a^-1 q_b)) (spherical.py:58-62), angle differences of atan2 for the
  // unbounded revolute and planar joints (revolute.py:233-237, planar.py:70-76)
  auto knot_differences = [&](const double* xs) {
    const int npair = 2 * T - 1;
    for (int e = tid; e < npair * nj; e += NT) {
      const int pi = divj.div(e), j = e - pi * nj;
      const int jt = jtype[j], nvj = joint_nv(jt);
      if (nvj == 0) continue;
      const int iq = idxq[j], iv = idxv[j];
      // configurations a -> b of the pair: (x_t, x_{t+1}) or (xref_t, x_t)
      const bool ref = pi >= T - 1;
      const int t = ref ? pi - (T - 1) : pi;
      const double* qbp = xs + (ref ? t : t + 1) * nq + iq;
      const double* qap = xs + t * nq + iq;
      const float* qrp = xref + t * nq + iq;
      auto qa = [&](int k) -> double { return ref ? (double)qrp[k] : qap[k]; };
      auto qb = [&](int k) -> double { return qbp[k]; };
      double* out = (ref ? dr : dd) + t * nv;
      if (jt == BR_JOINT_FREE_FLYER) {
        const DPose a{d3(qa(0), qa(1), qa(2)), make_double4(qa(3), qa(4), qa(5), qa(6))};
        const DPose b{d3(qb(0), qb(1), qb(2)), make_double4(qb(3), qb(4), qb(5), qb(6))};
        double3 v, w;
        dse3_log(dcompose(dinverse(a), b), v, w);
        out[iv] = v.x; out[iv + 1] = v.y; out[iv + 2] = v.z;
        out[iv + 3] = w.x; out[iv + 4] = w.y; out[iv + 5] = w.z;
      } else if (jt == BR_JOINT_SPHERICAL) {
        const double3 w = dso3_log(dqnormalize(dqmul(dqconj(make_double4(qa(0), qa(1), qa(2), qa(3))),
                                                     make_double4(qb(0), qb(1), qb(2), qb(3)))));
        out[iv] = w.x; out[iv + 1] = w.y; out[iv + 2] = w.z;
      } else if (jt == BR_JOINT_PLANAR || jt == BR_JOINT_REVOLUTE_UNBOUNDED) {
        const int k = jt == BR_JOINT_PLANAR ? 2 : 0;
        if (k) { out[iv] = qb(0) - qa(0); out[iv + 1] = qb(1) - qa(1); }
        out[iv + k] = atan2(qb(k + 1), qb(k)) - atan2(qa(k + 1), qa(k));
      } else {
        for (int k = 0; k < nvj; ++k) out[iv + k] = qb(k) - qa(k);
      }
    }
    __syncthreads();
  };
  // xn_t = integrate(x_t, delta_t) per knot (model.py:160-174): free-flyer normalize(q . exp(v))
  // (free_flyer.py:47-51), spherical normalize(q . exp(w)) (spherical.py:52-56), unbounded
  // revolute / planar angle atan2(s, c) + v as (cos, sin) (revolute.py:223-231, planar.py:61-68)
  auto retract_knots = [&]() {
    for (int e = tid; e < T * nj; e += NT) {
      const int t = divj.div(e), j = e - t * nj;
      const int jt = jtype[j], nvj = joint_nv(jt);
      if (nvj == 0) continue;
      const int iq = idxq[j], iv = idxv[j];
      const double* q = x + t * nq;
      const double* dv = delta + t * nv;
      double* o = xn + t * nq;
      if (jt == BR_JOINT_FREE_FLYER) {
        const DPose a{d3(q[iq], q[iq + 1], q[iq + 2]), make_double4(q[iq + 3], q[iq + 4], q[iq + 5], q[iq + 6])};
        DPose b = dcompose(a, dse3_exp(d3(dv[iv], dv[iv + 1], dv[iv + 2]), d3(dv[iv + 3], dv[iv + 4], dv[iv + 5])));
        b.q = dqnormalize(b.q);
        o[iq] = b.t.x; o[iq + 1] = b.t.y; o[iq + 2] = b.t.z;
        o[iq + 3] = b.q.x; o[iq + 4] = b.q.y; o[iq + 5] = b.q.z; o[iq + 6] = b.q.w;
      } else if (jt == BR_JOINT_SPHERICAL) {
        const double4 r = dqnormalize(dqmul(make_double4(q[iq], q[iq + 1], q[iq + 2], q[iq + 3]),
                                            dse3_exp(d3(0.0, 0.0, 0.0), d3(dv[iv], dv[iv + 1], dv[iv + 2])).q));
        o[iq] = r.x; o[iq + 1] = r.y; o[iq + 2] = r.z; o[iq + 3] = r.w;
      } else if (jt == BR_JOINT_PLANAR || jt == BR_JOINT_REVOLUTE_UNBOUNDED) {
        const int k = jt == BR_JOINT_PLANAR ? 2 : 0;
        if (k) { o[iq] = q[iq] + dv[iv]; o[iq + 1] = q[iq + 1] + dv[iv + 1]; }
        double sn, cs;
        sincos(atan2(q[iq + k + 1], q[iq + k]) + dv[iv + k], &sn, &cs);
        o[iq + k] = cs;
        o[iq + k + 1] = sn;
      } else {
        for (int k = 0; k < nvj; ++k) o[iq + k] = q[iq + k] + dv[iv + k];
      }
    }
  };
  // total cost 0.5 |r|^2 at xs (pose terms evaluated into rg / rs)
  auto cost_of = [&](const double* xs) -> double {
    double acc = 0.0;
    pose_terms(xs, false, false);
    if (kManifold) knot_differences(xs);
    for (int e = tid; e < (T - 2) * nv; e += NT) {              // smoothness.py:118-125
      const double a = kManifold ? c * (dd[e + nv] - dd[e]) : c * (xs[e + 2 * nv] - 2.0 * xs[e + nv] + xs[e]);
      acc += a * a;
    }
    if (kManifold) {
      for (int e = tid; e < nqT; e += NT) {                     // limits.py:56-62
        const int i = divq.mod(e);
        const double lo = fmax((double)lower[i] - xs[e], 0.0), hi = fmax(xs[e] - (double)upper[i], 0.0);
        acc += wl * wl * (lo * lo + hi * hi);
      }
      for (int e = tid; e < n; e += NT) acc += wr * wr * dr[e] * dr[e];   // regularization.py:143-152
    } else {                                                    // nq == nv: one pass for both
      for (int e = tid; e < n; e += NT) {
        const int i = divv.mod(e);
        const double lo = fmax((double)lower[i] - xs[e], 0.0), hi = fmax(xs[e] - (double)upper[i], 0.0);
        const double d = xs[e] - (double)xref[e];
        acc += wl * wl * (lo * lo + hi * hi) + wr * wr * d * d;
      }
    }
    acc = block_sum(acc);
    double pc = 0.0;
    for (int k = 0; k < 6; ++k) {
      if (has_goal) pc += wg * wg * rg[k] * rg[k];
      if (has_start) pc += ws * ws * rs[k] * rs[k];
    }
    return 0.5 * (acc + pc);
  };
  // J^T J of the pose terms (packed lower) and g = J^T r at x; returns |g|
  auto build = [&]() -> double {
    pose_terms(x, true, true);                        // FK and xi of x from the cost evaluation of x
    const int npk = nv * (nv + 1) / 2;
    for (int e = tid; e < npk; e += NT) {
      const int2 ab = tri_decode(e);
      double a = 0.0, b = 0.0;
      for (int r = 0; r < 6; ++r) {
        if (has_goal) a += Jg[r * nv + ab.x] * Jg[r * nv + ab.y];
        if (has_start) b += Js[r * nv + ab.x] * Js[r * nv + ab.y];
      }
      jtjg[e] = wg * wg * a;
      jtjs[e] = ws * ws * b;
    }
    double gg = 0.0;
    for (int e = tid; e < n; e += NT) {
      const int t = divv.div(e), i = e - t * nv;
      double acc = 0.0;
      // acceleration rows s = t, t-1, t-2 with coefficients +1, -2, +1 at knot t (the
      // identity-Jacobian blocks of smoothness.py:127-142)
      auto arow = [&](int s) {
        return kManifold ? c * (dd[(s + 1) * nv + i] - dd[s * nv + i])
                         : c * (x[(s + 2) * nv + i] - 2.0 * x[(s + 1) * nv + i] + x[s * nv + i]);
      };
      if (t <= T - 3) acc += c * arow(t);
      if (t - 1 >= 0 && t - 1 <= T - 3) acc += -2.0 * c * arow(t - 1);
      if (t - 2 >= 0) acc += c * arow(t - 2);
      const int iq = kManifold ? dofq[i] : i;
      if (iq >= 0) {
        const double xq = x[t * nq + iq];
        if (xq < (double)lower[iq]) acc -= wl * wl * ((double)lower[iq] - xq);
        if (xq > (double)upper[iq]) acc += wl * wl * (xq - (double)upper[iq]);
      }
      acc += wr * wr * (kManifold ? dr[e] : x[e] - (double)xref[e]);
      if (has_goal && t == T - 1)
        for (int r = 0; r < 6; ++r) acc += wg * wg * Jg[r * nv + i] * rg[r];
      if (has_start && t == 0)
        for (int r = 0; r < 6; ++r) acc += ws * ws * Js[r * nv + i] * rs[r];
      g[e] = acc;
      gg += acc * acc;
    }
    gg = block_sum(gg);
    return sqrt(gg);
  };
  // bands of J^T J + damp I at x (DOF i): diagonal at knot t, H[(t+1,i),(t,i)], and
  // H[(t+2,i),(t,i)] = c2 for t <= T-3.  Acceleration row s has coefficients (1, -2, 1)
  // on knots (s, s+1, s+2), s = 0..T-3.
  auto hdiag = [&](int t, int i, double damp) -> double {
    double a = 0.0;
    if (t <= T - 3) a += 1.0;
    if (t - 1 >= 0 && t - 1 <= T - 3) a += 4.0;
    if (t - 2 >= 0) a += 1.0;
    double d = c2 * a + wr * wr + damp;
    const int iq = kManifold ? dofq[i] : i;
    if (iq >= 0) {
      const double xv = x[t * nq + iq];
      if (xv < (double)lower[iq]) d += wl * wl;
      if (xv > (double)upper[iq]) d += wl * wl;
    }
    return d;
  };
  auto hoff1 = [&](int t) -> double {
    double b = 0.0;
    if (t <= T - 3) b += -2.0;
    if (t - 1 >= 0 && t <= T - 2) b += -2.0;
    return c2 * b;
  };
  // interior columns of the boundary knots: h0 = H[(t, i), (0, i)], hT = H[(t, i), (T-1, i)]
  auto h0_at = [&](int t) -> double { return t == 1 ? hoff1(0) : (t == 2 ? c2 : 0.0); };
  auto hT_at = [&](int t) -> double { return t == T - 2 ? hoff1(T - 2) : (t == T - 3 ? c2 : 0.0); };
  // solve (J^T J + damp I) delta = -g; false when a pivot is not positive.
  // Interior knots 1..T-2 of DOF i form the pentadiagonal P_i = L D L^T (thread i).  With
  // z = L^-1 v, the Schur complement terms are h^T P_i^-1 k = sum_p z_h[p] z_k[p] / D[p], so
  // one forward pass gives S = H_bb - H_bI P^-1 H_Ib and rb = -g_b - H_bI P^-1 (-g_I) without
  // storing P^-1 h0 and P^-1 hT; after the boundary solve, the interior step is one more
  // banded solve with right-hand side -g_I - h0 delta_0 - hT delta_{T-1}.
  // Twisted factorization (m = T - 2 >= kTwistMin interior knots): the band of DOF i is
  // factored from both ends at once, thread 2i taking rows 0..k-1 top-down (L D L^T) and
  // thread 2i + 1 rows m-1..k+2 bottom-up (U E U^T), k = m / 2, which halves the dependent
  // chain; both then reduce the 2 x 2 block of rows k, k+1 from the two sides' updates.  The
  // multipliers of the rows into the middle block are kept in the free slots of rows k, k+1
  // (bl1), every second-neighbour multiplier is c2 times a stored reciprocal pivot.  With
  // z = M^-1 v the twisted forward substitution, h^T P^-1 v is the sum over the top and bottom
  // rows of z_h z_v / pivot plus the middle block's r_h^T B^-1 r_v.
  constexpr int kTwistMin = 8;
  auto newton_solve = [&](double damp) -> bool {
    const int m = T - 2;
    const bool tw = m >= kTwistMin;
    const int km = m / 2;
    bool good = true;
    double suu = 0.0, suw = 0.0, sww = 0.0, suy = 0.0, swy = 0.0;
    const double h1 = -4.0 * c2;                    // H[(p+1), (p)] inside the interior
    if (!tw && tid < nv) {
      const int i = tid;
      double d1 = 0.0, di1 = 0.0, di2 = 0.0, l1p = 0.0;
      double y1 = 0, y2 = 0, u1 = 0, u2 = 0, w1 = 0, w2 = 0;
      for (int p = 0; p < m; ++p) {
        const int t = p + 1;
        const double l2 = (p >= 2) ? c2 * di2 : 0.0;
        const double l1 = (p >= 1) ? (h1 - c2 * l1p) * di1 : 0.0;
        const double dp = hdiag(t, i, damp) - l1 * l1 * d1 - l2 * c2;
        if (!(dp > 0.0)) { good = false; break; }
        const double dip = fast_rcp(dp);
        bl1[p * nv + i] = l1; bdi[p * nv + i] = dip;
        const double y = -g[t * nv + i] - l1 * y1 - l2 * y2;
        const double u = h0_at(t) - l1 * u1 - l2 * u2;
        const double w = hT_at(t) - l1 * w1 - l2 * w2;
        suu += u * u * dip; suw += u * w * dip; sww += w * w * dip;
        suy += u * y * dip; swy += w * y * dip;
        di2 = di1; di1 = dip; d1 = dp; l1p = l1;
        y2 = y1; y1 = y; u2 = u1; u1 = u; w2 = w1; w1 = w;
      }
    }
    const unsigned tmask = __ballot_sync(0xffffffffu, tid < 2 * nv);
    if (tw && tid < 2 * nv) {
      const int i = tid >> 1, side = tid & 1;
      // side 0: p = 0, 1, .., km-1; side 1: p = m-1, m-2, .., km+2 (the same recurrence on
      // the reversed band: diagonal, off-diagonals h1 and c2 are symmetric)
      const int p0 = side ? m - 1 : 0, dir = side ? -1 : 1, steps = side ? m - km - 2 : km;
      double d1 = 0.0, di1 = 0.0, di2 = 0.0, l1p = 0.0;
      double y1 = 0, y2 = 0, u1 = 0, u2 = 0, w1 = 0, w2 = 0;
      for (int q = 0; q < steps; ++q) {
        const int p = p0 + dir * q, t = p + 1;
        const double l2 = (q >= 2) ? c2 * di2 : 0.0;
        const double l1 = (q >= 1) ? (h1 - c2 * l1p) * di1 : 0.0;
        const double dp = hdiag(t, i, damp) - l1 * l1 * d1 - l2 * c2;
        if (!(dp > 0.0)) { good = false; break; }
        const double dip = fast_rcp(dp);
        bl1[p * nv + i] = l1; bdi[p * nv + i] = dip;
        const double y = -g[t * nv + i] - l1 * y1 - l2 * y2;
        const double u = h0_at(t) - l1 * u1 - l2 * u2;
        const double w = hT_at(t) - l1 * w1 - l2 * w2;
        suu += u * u * dip; suw += u * w * dip; sww += w * w * dip;
        suy += u * y * dip; swy += w * y * dip;
        di2 = di1; di1 = dip; d1 = dp; l1p = l1;
        y2 = y1; y1 = y; u2 = u1; u1 = u; w2 = w1; w1 = w;
      }
      // this side's multipliers into the middle block: the adjacent middle row (km for the top,
      // km + 1 for the bottom) from this side's last two rows, the far middle row from its last
      const double n1 = (h1 - c2 * l1p) * di1, n2 = c2 * di2, f1 = c2 * di1;
      const int near = side ? km + 1 : km;
      bl1[near * nv + i] = n1;
      // updates of the middle block: near diagonal, off-diagonal, far diagonal; right-hand sides
      const double a_near = n1 * n1 * d1 + n2 * c2, a_off = c2 * n1, a_far = f1 * c2;
      const double ry_near = n1 * y1 + n2 * y2, ry_far = f1 * y1;
      const double ru_near = n1 * u1 + n2 * u2, ru_far = f1 * u1;
      const double rw_near = n1 * w1 + n2 * w2, rw_far = f1 * w1;
      // the other side's updates (lanes 2i, 2i + 1 of one warp)
      const double o_near = __shfl_xor_sync(tmask, a_near, 1), o_off = __shfl_xor_sync(tmask, a_off, 1),
                   o_far = __shfl_xor_sync(tmask, a_far, 1);
      const double oy_near = __shfl_xor_sync(tmask, ry_near, 1), oy_far = __shfl_xor_sync(tmask, ry_far, 1);
      const double ou_near = __shfl_xor_sync(tmask, ru_near, 1), ou_far = __shfl_xor_sync(tmask, ru_far, 1);
      const double ow_near = __shfl_xor_sync(tmask, rw_near, 1), ow_far = __shfl_xor_sync(tmask, rw_far, 1);
      const double osuu = __shfl_xor_sync(tmask, suu, 1), osuw = __shfl_xor_sync(tmask, suw, 1),
                   osww = __shfl_xor_sync(tmask, sww, 1), osuy = __shfl_xor_sync(tmask, suy, 1),
                   oswy = __shfl_xor_sync(tmask, swy, 1);
      good = good && __shfl_xor_sync(tmask, (int)good, 1);
      // middle block in (top, bottom) order, the same on both lanes
      const double tA = side ? o_near : a_near, tF = side ? o_far : a_far, tO = side ? o_off : a_off;
      const double bA = side ? a_near : o_near, bF = side ? a_far : o_far, bO = side ? a_off : o_off;
      const int t0 = km + 1, t1 = km + 2;
      const double B00 = hdiag(t0, i, damp) - tA - bF;
      const double B10 = h1 - tO - bO;
      const double B11 = hdiag(t1, i, damp) - tF - bA;
      auto mid = [&](double v0, double v1, double top_near, double top_far, double bot_near, double bot_far,
                     double& r0, double& r1) {
        r0 = v0 - top_near - bot_far;
        r1 = v1 - top_far - bot_near;
      };
      double ry0, ry1, ru0, ru1, rw0, rw1;
      mid(-g[t0 * nv + i], -g[t1 * nv + i], side ? oy_near : ry_near, side ? oy_far : ry_far,
          side ? ry_near : oy_near, side ? ry_far : oy_far, ry0, ry1);
      mid(h0_at(t0), h0_at(t1), side ? ou_near : ru_near, side ? ou_far : ru_far,
          side ? ru_near : ou_near, side ? ru_far : ou_far, ru0, ru1);
      mid(hT_at(t0), hT_at(t1), side ? ow_near : rw_near, side ? ow_far : rw_far,
          side ? rw_near : ow_near, side ? rw_far : ow_far, rw0, rw1);
      good = good && B00 > 0.0;
      const double dk = good ? fast_rcp(B00) : 0.0;
      const double lm = B10 * dk;
      const double D1 = B11 - lm * B10;
      good = good && D1 > 0.0;
      const double dk1 = good ? fast_rcp(D1) : 0.0;
      if (side == 0) { bdi[km * nv + i] = dk; bdi[(km + 1) * nv + i] = dk1; }
      // a^T B^-1 b = a0 b0 / B00 + (a1 - l a0)(b1 - l b0) / D1
      auto bq = [&](double a0, double a1, double b0, double b1) {
        return a0 * b0 * dk + (a1 - lm * a0) * (b1 - lm * b0) * dk1;
      };
      suu += osuu + bq(ru0, ru1, ru0, ru1);
      suw += osuw + bq(ru0, ru1, rw0, rw1);
      sww += osww + bq(rw0, rw1, rw0, rw1);
      suy += osuy + bq(ru0, ru1, ry0, ry1);
      swy += oswy + bq(rw0, rw1, ry0, ry1);
    }
    if (__syncthreads_or(!good)) return false;
    // boundary block H_bb, packed lower: b = i for (knot 0, DOF i), nv + i for (knot T-1, DOF i)
    const int nbp = nb * (nb + 1) / 2;
    for (int e = tid; e < nbp; e += NT) {
      const int2 rc = tri_decode(e);
      const int r = rc.x, cc = rc.y;
      const int kr = r >= nv, kc = cc >= nv, ir = r - kr * nv, ic = cc - kc * nv;
      double h = 0.0;
      if (kr == kc) {
        const int pe = ir >= ic ? tri_at(ir, ic) : tri_at(ic, ir);
        if (kr == 0 && has_start) h = jtjs[pe];
        if (kr == 1 && has_goal) h = jtjg[pe];
        if (ir == ic) h += hdiag(kr ? T - 1 : 0, ir, damp);
      } else if (ir == ic && T == 3) {
        h = c2;                                                    // row 0 couples knots 0 and 2
      }
      Sb[e] = h;
    }
    __syncthreads();
    if (tw ? (tid < 2 * nv && (tid & 1) == 0) : tid < nv) {
      const int i = tw ? tid >> 1 : tid;
      Sb[tri_at(i, i)] -= suu;
      Sb[tri_at(nv + i, i)] -= suw;
      Sb[tri_at(nv + i, nv + i)] -= sww;
      rb[i] = -g[i] - suy;
      rb[nv + i] = -g[(T - 1) * nv + i] - swy;
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {                                  // chol(S), lower, in place
      const double dkk = Sb[tri_at(k, k)];
      if (!(dkk > 0.0)) return false;                               // every thread read the same value
      const double inv = fast_rsqrt(dkk);
      __syncthreads();
      for (int r = k + 1 + tid; r < nb; r += NT) Sb[tri_at(r, k)] *= inv;
      if (tid == 0) { Sb[tri_at(k, k)] = dkk * inv; sdi[k] = inv; }
      __syncthreads();
      // trailing update S[r][cc] -= L[r][k] L[cc][k], k < cc <= r < nb, as packed pairs
      const int np = (nb - k - 1) * (nb - k) / 2;
      for (int pp = tid; pp < np; pp += NT) {
        const int2 ab = tri_decode(pp);
        const int r = ab.x + k + 1, cc = ab.y + k + 1;
        Sb[tri_at(r, cc)] -= Sb[tri_at(r, k)] * Sb[tri_at(cc, k)];
      }
      __syncthreads();
    }
    // z = S^-1 rb
    if (nb <= kWarp) {
      if (warp == 0) {                      // lane b owns entry b; one finished entry broadcast per step
        double v = (lane < nb) ? rb[lane] : 0.0;
        for (int j = 0; j < nb; ++j) {
          const double zj = __shfl_sync(0xffffffffu, v, j) * sdi[j];
          if (lane == j) v = zj;
          else if (lane > j && lane < nb) v -= Sb[tri_at(lane, j)] * zj;
        }
        for (int j = nb - 1; j >= 0; --j) {
          const double zj = __shfl_sync(0xffffffffu, v, j) * sdi[j];
          if (lane == j) v = zj;
          else if (lane < j) v -= Sb[tri_at(j, lane)] * zj;
        }
        if (lane < nb) zb[lane] = v;
      }
    } else {                                // column-oriented substitutions over the block
      for (int j = 0; j < nb; ++j) {        // L y = rb (rb overwritten by the partial sums)
        const double yj = rb[j] * sdi[j];
        for (int r = j + 1 + tid; r < nb; r += NT) rb[r] -= Sb[tri_at(r, j)] * yj;
        if (tid == 0) zb[j] = yj;
        __syncthreads();
      }
      for (int j = nb - 1; j >= 0; --j) {   // L^T z = y (zb overwritten in place)
        const double zj = zb[j] * sdi[j];
        __syncthreads();
        for (int r = tid; r < j; r += NT) zb[r] -= Sb[tri_at(j, r)] * zj;
        if (tid == 0) zb[j] = zj;
        __syncthreads();
      }
    }
    __syncthreads();
    // interior step of DOF i: P_i d = -g_I - h0 z(knot 0) - hT z(knot T-1); forward into delta,
    // then backward in place (twisted: from both ends to the middle block and back out)
    if (tw && tid < 2 * nv) {
      const int i = tid >> 1, side = tid & 1;
      const double z0 = zb[i], zT = zb[nv + i];
      if (side == 0) {
        delta[i] = z0;
        delta[(T - 1) * nv + i] = zT;
      }
      auto rhs = [&](int t) { return -g[t * nv + i] - h0_at(t) * z0 - hT_at(t) * zT; };
      const int p0 = side ? m - 1 : 0, dir = side ? -1 : 1, steps = side ? m - km - 2 : km;
      double y1 = 0, y2 = 0;
      for (int q = 0; q < steps; ++q) {
        const int p = p0 + dir * q, t = p + 1;
        const double l1 = bl1[p * nv + i], l2 = (q >= 2) ? c2 * bdi[(p - 2 * dir) * nv + i] : 0.0;
        const double y = rhs(t) - l1 * y1 - l2 * y2;
        delta[t * nv + i] = y;
        y2 = y1; y1 = y;
      }
      // middle block: this side's last two rows, multipliers as in the factorization
      const int pl = p0 + dir * (steps - 1);                      // this side's last row
      const double n1 = bl1[(side ? km + 1 : km) * nv + i];
      const double n2 = c2 * bdi[(pl - dir) * nv + i], f1 = c2 * bdi[pl * nv + i];
      const double r_near = n1 * y1 + n2 * y2, r_far = f1 * y1;
      const double o_near = __shfl_xor_sync(tmask, r_near, 1), o_far = __shfl_xor_sync(tmask, r_far, 1);
      const double on1 = __shfl_xor_sync(tmask, n1, 1);
      const double tn = side ? o_near : r_near, tf = side ? o_far : r_far;
      const double bn = side ? r_near : o_near, bfar = side ? r_far : o_far;
      const double r0 = rhs(km + 1) - tn - bfar, r1 = rhs(km + 2) - tf - bn;
      const double dk = bdi[km * nv + i], dk1 = bdi[(km + 1) * nv + i];
      const double lm = (h1 - c2 * n1 - c2 * on1) * dk;           // B10 / B00 (symmetric in the sides)
      const double x1 = (r1 - lm * r0) * dk1, x0 = r0 * dk - lm * x1;
      if (side == 0) {
        delta[(km + 1) * nv + i] = x0;
        delta[(km + 2) * nv + i] = x1;
      }
      // back substitution outwards: x_p = z_p / pivot_p - (near multiplier) x_(p+dir') - c2 / pivot_p x_(p+2dir')
      double xa = side ? x1 : x0, xb = side ? x0 : x1;            // the next two rows towards the middle
      for (int q = steps - 1; q >= 0; --q) {
        const int p = p0 + dir * q;
        const double di = bdi[p * nv + i];
        const double ln = bl1[(p + dir) * nv + i];                 // the row towards the middle, relative to p
        const double y = delta[(p + 1) * nv + i] * di - ln * xa - c2 * di * xb;
        delta[(p + 1) * nv + i] = y;
        xb = xa; xa = y;
      }
    }
    if (!tw && tid < nv) {
      const int i = tid;
      const double z0 = zb[i], zT = zb[nv + i];
      delta[i] = z0;
      delta[(T - 1) * nv + i] = zT;
      double y1 = 0, y2 = 0;
      for (int p = 0; p < m; ++p) {
        const int t = p + 1;
        const double l1 = bl1[p * nv + i], l2 = (p >= 2) ? c2 * bdi[(p - 2) * nv + i] : 0.0;
        const double y = -g[t * nv + i] - h0_at(t) * z0 - hT_at(t) * zT - l1 * y1 - l2 * y2;
        delta[t * nv + i] = y;
        y2 = y1; y1 = y;
      }
      y1 = y2 = 0;
      for (int p = m - 1; p >= 0; --p) {
        const double di = bdi[p * nv + i];
        const double l1n = (p + 1 < m) ? bl1[(p + 1) * nv + i] : 0.0;   // L[p+1][p]
        const double l2n = (p + 2 < m) ? c2 * di : 0.0;                  // L[p+2][p] = c2 / D[p]
        const double y = delta[(p + 1) * nv + i] * di - l1n * y1 - l2n * y2;
        delta[(p + 1) * nv + i] = y;
        y2 = y1; y1 = y;
      }
    }
    __syncthreads();
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
    if (!newton_solve(lm ? lam : (double)S.gn_eps)) {
      flags |= BR_IK_FLAG_REGULARIZED;
      bool ok = false;
      double extra = 1e-9;
      for (int k = 0; k < 8 && !ok; ++k, extra *= 10.0) {
        ok = newton_solve((lm ? lam : (double)S.gn_eps) + extra);
      }
      if (!ok) {
        for (int e = tid; e < n; e += NT) delta[e] = 0.0;
        __syncthreads();
      }
    }
    if (kManifold) {                                               // Model.integrate per knot (trajopt.py:159-169)
      retract_knots();
    } else {
      for (int e = tid; e < n; e += NT) xn[e] = x[e] + delta[e];
    }
    __syncthreads();
    const double cn = cost_of(xn);
    if (!isfinite(cn)) flags |= BR_IK_FLAG_NONFINITE;
    bool accept = !lm || cn < cost;
    if (accept) {
      for (int e = tid; e < nqT; e += NT) x[e] = xn[e];
      __syncthreads();
      cost = cn;
      need = true;
      if (lm) lam = fmax(lam / S.factor, (double)S.lam_min);
      if (gnorm < S.tol) { status = BR_IK_CONVERGED; ++it; break; }
    } else {
      lam = fmin(lam * S.factor, (double)S.lam_max);
    }
  }
  float* xo = P.x + traj * (int64_t)nqT;
  for (int e = tid; e < nqT; e += NT) xo[e] = (float)x[e];
  if (P.goal_grad && has_goal) {
    pose_terms(x, false, false);
    __syncthreads();
    if (tid == 0) {
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
  if (tid == 0) {
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
  {
    const int ok = (1 << (BR_JOINT_TRANSLATION + 1)) - 1;        // every kind of the tree table
    if (tree->kinds == 0 || (tree->kinds & ~ok)) return BR_EINVAL;
  }
  const int manifold_kinds = (1 << BR_JOINT_FREE_FLYER) | (1 << BR_JOINT_SPHERICAL) | (1 << BR_JOINT_PLANAR) |
                             (1 << BR_JOINT_REVOLUTE_UNBOUNDED);
  if (!(tree->kinds & manifold_kinds) && tree->nq != tree->nv) return BR_EINVAL;
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
  const bool floating = (tree->kinds & manifold_kinds) != 0;
  const TrajLayout L(tree->njoints, tree->nq, tree->nv, knots, floating);
  const size_t bytes = (size_t)L.total * sizeof(double);
  const DeviceInfo& dev = device_info();
  if ((int64_t)bytes > dev.max_smem_optin) return BR_ETOOBIG;
  auto kern = floating ? traj_gn_kernel<true> : traj_gn_kernel<false>;
  static int configured[2][16] = {{0}};
  int& conf = configured[floating ? 1 : 0][dev.device & 15];
  if ((int)bytes > conf) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    conf = (int)bytes;
  }
  if (n_traj > 0x7fffffff) return BR_ETOOBIG;
  kern<<<(unsigned)n_traj, kTrajThreads, bytes, (cudaStream_t)stream>>>(p);
  return (int)cudaGetLastError();
}

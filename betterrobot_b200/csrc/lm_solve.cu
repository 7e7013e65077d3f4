// lm_solve.cu — persistent batched Levenberg-Marquardt / Gauss-Newton IK for sm_100a.
//
// One launch solves thousands of independent IK problems of uneven size
// (different robots, DOF and target counts).  The reference solves one problem
// per call with >= 3 host syncs per iteration
// (src/better_robot/optim/optimizers/levenberg_marquardt.py:61-135); here the whole
// loop stays on the device:
//
//   * a TEAM of T = 32 lanes (one warp) owns one problem; warps take problems from
//     an atomic queue, heaviest robot class first.  A warp whose problem converges
//     leaves the loop and takes the next item, so no lane keeps iterating a
//     converged problem (work compaction by queue).  The team code is written for
//     any T in {8, 16, 32}; only T = 32 is instantiated (see lm_solve_kernel);
//   * per iteration: forward kinematics of the trial point by pointer jumping in
//     shared memory, the stacked residual (pose targets, joint limits, rest) and
//     its cost by a team reduction, accept/reject, and — only after an accepted
//     step, because the reference recomputes an identical J after a rejection —
//     the Jacobian build: J^T J and J^T r accumulated directly from the analytic
//     pose Jacobian Jr^-1(xi) blockdiag(R^T, R^T) J_lwa (pose.py:68-103) with columns
//     outside a target's support skipped;
//   * H = J^T J + lambda I, stored per DOF over its ancestors in the DOF tree,
//     factored leaves first as an unscaled LDL^T (no fill-in), all DOFs of one
//     height in the DOF tree at once (br_tree_t.dof_sched, built on the host by
//     br_dof_schedule), the right-hand side updated in the same tasks, back
//     substitution by depth with the right-hand sides in registers;
//   * retraction q (+) dq (Model.integrate, model.py:160-174) and clamping to the
//     joint limits (levenberg_marquardt.py:103-107).
//
// Precision: the iterate, forward kinematics, residual, cost and retraction are
// float64, so `cost_new < cost` (levenberg_marquardt.py:114) and the convergence
// test are decided as the float64 reference decides them; near the optimum the
// cost decrease of an accepted step (~1e-12) is far below float32 resolution of
// the cost.  Everything that scales with nv^2 or nv^3 — Jacobian columns, J^T J,
// J^T r, the Cholesky factorization and the solves — is float32, and so is the
// exponential of a free-flyer step in the plain variant (composed with the float64
// iterate in float64; its rounding is relative to the step).
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/br_b200.h"
#include "br_common.cuh"
#include "br_fk.cuh"
#include "br_lie.cuh"

namespace br {

constexpr int kMaxClasses = BR_MAX_IK_CLASSES;

struct LmParams {
  br_ik_settings_t s;
  br_ik_batch_t b;
  br_ik_result_t r;
  br_tree_t trees[kMaxClasses];
  int32_t team[kMaxClasses];
  int32_t warp_floats;       // per-warp shared memory (floats)
  int32_t* queue;            // scratch: work-queue counter (zeroed before launch)
};

// ---- per-team shared-memory layout (floats) --------------------------------
struct TeamLayout {
  int parent, jtype, idxq, idxv, support, cjoint, ckind, caxis, lower, upper;
  int fparent, fplace, tgt, tkind;
  int dpar, ddep, rowoff, amask, ancd;
  int x, xn, qrest, poseA, poseB, ancA, ancB, tw, xi, jri, colw, d, g, delta, jtj, work, misc,
      dinv, sup, nsup;
  int n_ent, anc_stride;  // capacity of the J^T J / factor storage; row length of ancd
  int total;
  // ent / dep: the tree's DOF entry count and depth bound (br_tree_t.dof_entries /
  // dof_depth), 0 for the dense bounds.
  // rounds: the tree's pointer-jumping FK rounds (br_tree_t.rounds), which decide the
  // pose buffer FK returns.
  // rs: floats per scalar of the Jacobian / normal-equation regions (1: float32, 2: float64).
  __host__ __device__ TeamLayout(int nj, int nq, int nv, int K, int T, int ent, int dep, int rounds, int rs = 1) {
    int o = 0;
    auto take = [&](int n) { int r = o; o += round4(n); return r; };
    parent = take(nj); jtype = take(nj); idxq = take(nj); idxv = take(nj);
    support = take(2 * nj);
    cjoint = take(nv); ckind = take(nv); caxis = take(4 * nv);
    lower = take(nq); upper = take(nq);
    fparent = take(K); fplace = take(8 * K); tkind = take(K);
    // float64 regions (2 floats per double)
    x = take(2 * nq); xn = take(2 * nq); qrest = take(2 * nq);
    poseA = take(14 * nj); poseB = take(14 * nj); tw = take(16 * K); xi = take(16 * K);
    d = take(2 * nv);
    tgt = take(16 * K);
    // normal-equation regions (rs floats per scalar), then float32 / int regions
    jri = take(16 * K * rs); colw = take(8 * nv * rs);
    g = take(nv * rs); delta = take(nv * rs);
    const int ntri = nv * (nv + 1) / 2;
    n_ent = (ent > 0 && ent < ntri) ? ent : ntri;
    anc_stride = (dep > 0 && dep < nv) ? dep : (nv > 0 ? nv : 1);
    jtj = take(n_ent * rs);                    // J^T J, one row per DOF over its ancestors
    // two targets' J columns (build) / the factor and its right-hand-side slots (solve):
    // in the pose buffer that FK does not return (poseA after an odd number of rounds, else
    // poseB), dead while the normal equations are built and solved, when it is large enough
    const int wneed = (12 * nv > n_ent + nv ? 12 * nv : n_ent + nv) * rs;
    work = wneed <= 14 * nj ? ((rounds & 1) ? poseA : poseB) : take(wneed);
    dinv = take(nv * rs);                      // 1 / L_jj
    ancA = take(nj); ancB = take(nj);
    misc = take(8);
    amask = take(2 * nv);                      // uint64 strict ancestors of each DOF
    dpar = take((nv + 3) / 4);                 // int8 parent DOF (-1 at a root)
    ddep = take((nv + 3) / 4);                 // uint8 DOF depth
    rowoff = take((nv + 2) / 2);               // uint16 first entry of each row, nv + 1 values
    ancd = take((nv * anc_stride + 3) / 4);    // uint8 ancestor of DOF c at depth a: ancd[c * anc_stride + a]
    sup = take((K * nv + 3) / 4);              // uint8 support columns of each target, ascending
    nsup = take(K);
    total = o;
  }
};

__device__ __forceinline__ int tri(int i) { return i * (i + 1) / 2; }
// Largest trunk (root chain above every other DOF) factored in registers by the float64
// variants: its ntr (ntr + 1) / 2 factor entries and ntr right-hand sides take one lane each
// of a 32-lane team.
constexpr int kTrunkMax = 6;


// IRLS weight w(s) of one squared residual row s (optim/kernels/{huber,cauchy,tukey}.py:
// weight; applied as in levenberg_marquardt.py:27-44, whose sqrt(w) scales both the row
// and its Jacobian row, so J^T J and J^T r pick up w).  Evaluated in float64.
template <typename R>
__device__ __forceinline__ R irls_weight(int kernel, double c, double s) {
  switch (kernel) {
    case BR_KERNEL_HUBER: return s <= c * c ? (R)1 : (R)(c / sqrt(fmax(s, 0.0) + 1e-30));
    case BR_KERNEL_CAUCHY: return (R)(1.0 / (1.0 + s / (c * c)));
    case BR_KERNEL_TUKEY: {
      const double u = fmax(1.0 - s / (c * c), 0.0);
      return (R)(u * u);
    }
    default: return (R)1;
  }
}

// Scalar helpers of the normal-equation arithmetic, for R = float (the default variant) or
// R = double (the float64 variant: the Jacobian, J^T J, J^T r and the factorization in float64).
__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float rrcp(float a) { return __frcp_rn(a); }
__device__ __forceinline__ double rrcp(double a) { return __drcp_rn(a); }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float rmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double rmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float rsqrt_(float a) { return sqrtf(a); }
__device__ __forceinline__ double rsqrt_(double a) { return sqrt(a); }

// C(th^2) of the SO3 Jr^-1 = I + W/2 + C W^2, C = 1/th^2 - (1 + cos th) / (2 th sin th)
// (tangents.py:122-145), in float64: its Taylor series 1/12 + th^2/720 + th^4/30240 +
// th^6/1209600 + th^8/47900160 below th^2 = 0.1 (the next term is below 1e-15 of C there),
// else the closed form.
__device__ __forceinline__ double dvinv_coeff(double th2) {
  if (th2 < 0.1) {
    return fma(th2, fma(th2, fma(th2, fma(th2, 1.0 / 47900160.0, 1.0 / 1209600.0), 1.0 / 30240.0), 1.0 / 720.0),
               1.0 / 12.0);
  }
  const double th = sqrt(th2);
  double s, c;
  sincos(th, &s, &c);
  return 1.0 / th2 - (1.0 + c) / (2.0 * th * s);
}

// Lanes per problem (team size) the kernel is built for, and the DOFs one lane owns in the
// register triangular solves (lm_rows(T) * T >= BR_MAX_NV).
constexpr int kLmTeam = 32;
__host__ __device__ constexpr int lm_rows(int T) { return (BR_MAX_NV + T - 1) / T; }

template <int T>
struct Team {
  unsigned mask;
  int tl;  // lane within team
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ float sum(float v) const {
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, T);
    return v;
  }
  __device__ __forceinline__ float bcast(float v, int src) const { return __shfl_sync(mask, v, src, T); }
};

__device__ __forceinline__ Pose ld8(const float* p) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  Pose P;
  P.t = f3(a.x, a.y, a.z);
  P.q = *reinterpret_cast<const float4*>(p + 4);
  return P;
}
__device__ __forceinline__ void st8(float* p, const Pose& P) {
  *reinterpret_cast<float4*>(p) = make_float4(P.t.x, P.t.y, P.t.z, 0.f);
  *reinterpret_cast<float4*>(p + 4) = P.q;
}

// float64 joint poses in structure-of-arrays form: 7 arrays of nj doubles
// (t.x, t.y, t.z, q.x, q.y, q.z, q.w), so lanes reading consecutive joints hit
// consecutive 8-byte words (no bank conflicts).
__device__ __forceinline__ DPose lds(const double* p, int nj, int j) {
  DPose P;
  P.t = d3(p[j], p[nj + j], p[2 * nj + j]);
  P.q = make_double4(p[3 * nj + j], p[4 * nj + j], p[5 * nj + j], p[6 * nj + j]);
  return P;
}
__device__ __forceinline__ void sts(double* p, int nj, int j, const DPose& P) {
  p[j] = P.t.x; p[nj + j] = P.t.y; p[2 * nj + j] = P.t.z;
  p[3 * nj + j] = P.q.x; p[4 * nj + j] = P.q.y; p[5 * nj + j] = P.q.z; p[6 * nj + j] = P.q.w;
}
// float64 per-target records: (t.x, t.y, t.z, pad, q.x, q.y, q.z, q.w)
__device__ __forceinline__ DPose ldd(const double* p) {
  DPose P;
  P.t = d3(p[0], p[1], p[2]);
  P.q = make_double4(p[4], p[5], p[6], p[7]);
  return P;
}
__device__ __forceinline__ void std8(double* p, const DPose& P) {
  p[0] = P.t.x; p[1] = P.t.y; p[2] = P.t.z; p[3] = 0.0;
  p[4] = P.q.x; p[5] = P.q.y; p[6] = P.q.z; p[7] = P.q.w;
}
__device__ __forceinline__ DPose to_d(const Pose& P) {
  return DPose{d3(P.t.x, P.t.y, P.t.z), make_double4(P.q.x, P.q.y, P.q.z, P.q.w)};
}
__device__ __forceinline__ Pose to_f(const DPose& P) {
  return Pose{f3((float)P.t.x, (float)P.t.y, (float)P.t.z),
              make_float4((float)P.q.x, (float)P.q.y, (float)P.q.z, (float)P.q.w)};
}

// ---- one problem, solved by one team ---------------------------------------
// kGeneral = false compiles the plain stack (pose targets, l2 kernel, fixed / revolute /
// prismatic / free-flyer joints) with the other branches folded away; the host launches it
// whenever a batch needs nothing else.
// kF64 = true computes the Jacobian columns, J^T J, J^T r, the factorization and the step in
// float64 (R = double) instead of float32.
template <int T, bool kGeneral, bool kF64>
__device__ void solve_problem(const LmParams& P, const br_tree_t& tree, int prob, float* sm, const Team<T>& tm,
                              const uint32_t*& sched_ok) {
  using R = typename std::conditional<kF64, double, float>::type;
  const int nj = tree.njoints, nq = tree.nq, nv = tree.nv;
  const int K = P.b.max_targets;
  const TeamLayout L(nj, nq, nv, K, T, tree.dof_entries, tree.dof_depth, tree.rounds, kF64 ? 2 : 1);
  int* parent = reinterpret_cast<int*>(sm + L.parent);
  int* jtype = reinterpret_cast<int*>(sm + L.jtype);
  int* idxq = reinterpret_cast<int*>(sm + L.idxq);
  int* idxv = reinterpret_cast<int*>(sm + L.idxv);
  const float* __restrict__ axis = tree.axis;         // read-only cache
  const float* __restrict__ place = tree.placement;
  unsigned long long* support = reinterpret_cast<unsigned long long*>(sm + L.support);
  int* cjoint = reinterpret_cast<int*>(sm + L.cjoint);
  int* ckind = reinterpret_cast<int*>(sm + L.ckind);
  float* caxis = sm + L.caxis;
  float* lower = sm + L.lower;
  float* upper = sm + L.upper;
  int* fparent = reinterpret_cast<int*>(sm + L.fparent);
  int* tkind = reinterpret_cast<int*>(sm + L.tkind);
  float* fplace = sm + L.fplace;
  double* x = reinterpret_cast<double*>(sm + L.x);
  double* xn = reinterpret_cast<double*>(sm + L.xn);
  double* qrest = reinterpret_cast<double*>(sm + L.qrest);
  double* poseA = reinterpret_cast<double*>(sm + L.poseA);
  double* poseB = reinterpret_cast<double*>(sm + L.poseB);
  double* tw = reinterpret_cast<double*>(sm + L.tw);
  double* xi = reinterpret_cast<double*>(sm + L.xi);
  double* dr = reinterpret_cast<double*>(sm + L.d);
  double* tgt = reinterpret_cast<double*>(sm + L.tgt);
  int* ancA = reinterpret_cast<int*>(sm + L.ancA);
  int* ancB = reinterpret_cast<int*>(sm + L.ancB);
  R* jri = reinterpret_cast<R*>(sm + L.jri);
  R* colw = reinterpret_cast<R*>(sm + L.colw);
  R* g = reinterpret_cast<R*>(sm + L.g);
  R* delta = reinterpret_cast<R*>(sm + L.delta);
  R* jtj = reinterpret_cast<R*>(sm + L.jtj);
  R* work = reinterpret_cast<R*>(sm + L.work);
  unsigned long long* amask = reinterpret_cast<unsigned long long*>(sm + L.amask);
  signed char* dpar = reinterpret_cast<signed char*>(sm + L.dpar);
  unsigned char* ddep = reinterpret_cast<unsigned char*>(sm + L.ddep);
  unsigned short* rowoff = reinterpret_cast<unsigned short*>(sm + L.rowoff);
  unsigned char* ancd = reinterpret_cast<unsigned char*>(sm + L.ancd);
  R* dinv = reinterpret_cast<R*>(sm + L.dinv);
  int* misc = reinterpret_cast<int*>(sm + L.misc);  // [0]: the tree's tables are inconsistent; [1]: 1 + max DOF depth
  unsigned char* sup = reinterpret_cast<unsigned char*>(sm + L.sup);
  int* nsup = reinterpret_cast<int*>(sm + L.nsup);
  const int tl = tm.tl;
  const br_ik_settings_t& S = P.s;
  const R wp = (R)S.pos_weight, wo = (R)S.ori_weight, wl = (R)S.limit_weight, wr = (R)S.rest_weight;
  const double wpd = wp, wod = wo, wld = wl, wrd = wr;
  const double kc = S.kernel_param;
  const bool irls = kGeneral && S.kernel != BR_KERNEL_L2;
  const bool use_limits = S.limit_weight > 0.f, use_rest = S.rest_weight > 0.f;
  // packed lower-triangle pair p -> (a, b), b <= a, p = tri(a) + b
  auto decode_pair = [](int p) {
    float r;  // approximate square root: the two corrections below make the decode exact
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(8.f * p + 1.f));
    int a = (int)((r - 1.f) * 0.5f);
    if (tri(a + 1) <= p) ++a;
    if (tri(a) > p) --a;
    return a | ((p - tri(a)) << 8);
  };

  // ---- load the tree table and the problem -------------------------------
#pragma unroll 1
  for (int j = tl; j < nj; j += T) {
    parent[j] = tree.parent[j];
    jtype[j] = tree.jtype[j];
    idxq[j] = tree.idx_q[j];
    idxv[j] = tree.idx_v[j];
    support[j] = tree.support[j];
  }
#pragma unroll 1
  for (int c = tl; c < nv; c += T) {
    cjoint[c] = tree.col_joint[c];
    ckind[c] = tree.col_kind[c];
    *reinterpret_cast<float4*>(caxis + 4 * c) = *reinterpret_cast<const float4*>(tree.col_axis + 4 * c);
  }
  const int64_t qoff = P.b.q_offset[prob];
#pragma unroll 1
  for (int i = tl; i < nq; i += T) {
    lower[i] = tree.lower[i];
    upper[i] = tree.upper[i];
    x[i] = (double)P.b.x0[qoff + i];
    qrest[i] = (double)P.b.q_rest[qoff + i];
  }
  const int nt = P.b.n_targets[prob];
  for (int t = tl; t < K; t += T) {
    if (t < nt) {
      const int f = P.b.frames[(int64_t)prob * K + t];
      fparent[t] = tree.frame_parent[f];
      tkind[t] = (kGeneral && P.b.target_kind) ? P.b.target_kind[(int64_t)prob * K + t] : BR_TARGET_POSE;
      for (int k = 0; k < 8; ++k) fplace[8 * t + k] = tree.frame_placement[8 * f + k];
      const float* tp = P.b.targets + ((int64_t)prob * K + t) * 7;
      std8(tgt + 8 * t, DPose{d3(tp[0], tp[1], tp[2]), make_double4(tp[3], tp[4], tp[5], tp[6])});
    }
  }
  // ---- the DOF tree of J^T J -----------------------------------------------
  // DOF c's parent is the previous DOF of its own joint (a free-flyer's 6 DOFs form a
  // chain) or the last DOF of the nearest ancestor joint that has DOFs.  The residuals
  // couple a DOF only with its ancestors (a pose target's support is a root-to-frame
  // path; limit, rest and damping terms are diagonal), so J^T J is stored as one row per
  // DOF over its ancestors and itself, entry (i, j) at rowoff[i] + ddep[j], and factors
  // leaves first with no fill-in.  DOF numbering is topological (dpar[c] < c), so a
  // DOF's ancestors have smaller indices.  One lane builds the tables once per problem.
  if (tl == 0) {
    int* lastd = reinterpret_cast<int*>(poseA);  // scratch: last DOF on each joint's path
    for (int j = 0; j < nj; ++j) {
      const int pj = parent[j];
      const int prev = pj >= 0 ? lastd[pj] : -1;
      const int jt = jtype[j];
      const int nvj = joint_nv(jt);
      for (int k = 0; k < nvj; ++k) dpar[idxv[j] + k] = (signed char)(k == 0 ? prev : idxv[j] + k - 1);
      lastd[j] = nvj ? idxv[j] + nvj - 1 : prev;
    }
    int nl = 0, dlev = 0;
    bool bad = false;
    const int As = L.anc_stride;
    for (int c = 0; c < nv; ++c) {
      const int pc = dpar[c];
      const int dc = pc < 0 ? 0 : ddep[pc] + 1;
      ddep[c] = (unsigned char)dc;
      dlev = dc + 1 > dlev ? dc + 1 : dlev;
      amask[c] = pc < 0 ? 0ull : (amask[pc] | (1ull << pc));
      if (dc > As) {
        bad = true;  // deeper than the tree's dof_depth claims: the ancestor table would overflow
      } else {
#pragma unroll 1
        for (int a = 0; a + 1 < dc; ++a) ancd[c * As + a] = ancd[pc * As + a];
        if (pc >= 0) ancd[c * As + dc - 1] = (unsigned char)pc;
      }
      rowoff[c] = (unsigned short)nl;
      nl += dc + 1;
    }
    rowoff[nv] = (unsigned short)nl;
    misc[0] = (bad || nl > L.n_ent) ? 1 : 0;
    misc[1] = dlev;
    // trunk: the largest n <= kTrunkMax such that DOFs 0..n-1 form a chain from the root and
    // every other DOF descends from DOF n - 1 (a floating base's six DOFs; the top of a serial
    // chain).  The schedule's last n levels then eliminate n - 1, ..., 0, one DOF each.
    int ntr = 0;
#pragma unroll 1
    for (int n = kF64 ? (nv < kTrunkMax ? nv : kTrunkMax) : 0; n >= 2 && ntr == 0; --n) {
      bool ok = dpar[0] < 0;
#pragma unroll 1
      for (int c = 1; c < n && ok; ++c) ok = dpar[c] == c - 1;
#pragma unroll 1
      for (int c = n; c < nv && ok; ++c) ok = ((amask[c] >> (n - 1)) & 1ull) != 0;
      if (ok) ntr = n;
    }
    misc[2] = ntr;
  }
  tm.sync();
  // level schedule (br_tree_t.dof_sched): every offset it holds must address this
  // problem's factor storage; checked once per team and schedule
  const uint32_t* sched = tree.dof_sched;  // non-null: checked on the host
  if (sched != sched_ok && !misc[0]) {
    const int nL0 = rowoff[nv], lim = nL0 + nv;
    const int nlev = (int)sched[0], ntask = (int)sched[1], nextra = (int)sched[2];
    bool bad = nlev < 0 || nlev > nv || ntask < 0 || nextra < 0 || (int)sched[3] != misc[1];
    if (!bad) {
#pragma unroll 1
      for (int l = tl; l <= nlev; l += T) {
        const int s0 = (int)sched[4 + l];
        bad |= (l == 0 && s0 != 0) || (l == nlev && s0 != ntask) || s0 < 0 || s0 > ntask ||
               (l > 0 && s0 < (int)sched[3 + l]);
      }
      const int toff = (5 + nlev + 3) & ~3;
      const uint4* tk = reinterpret_cast<const uint4*>(sched + toff);
      const uint2* ex = reinterpret_cast<const uint2*>(sched + toff + 4 * ntask);
      for (int p = tl; p < ntask; p += T) {
        const uint4 t4 = tk[p];
        bad |= (int)(t4.x & 0xffff) >= lim || (int)(t4.y & 0xffff) >= lim || (int)(t4.y >> 16) >= lim ||
               (int)(t4.z & 0xffff) >= nv || (int)(t4.z >> 16) + (int)(t4.x >> 16) > nextra || (int)t4.w > nv;
      }
#pragma unroll 1
      for (int e = tl; e < nextra; e += T) {
        const uint2 e2 = ex[e];
        bad |= (int)(e2.x & 0xffff) >= lim || (int)(e2.x >> 16) >= lim || (int)e2.y >= nv;
      }
    }
    bad = __any_sync(tm.mask, bad);
    if (bad) {
      if (tl == 0) misc[0] = 1;
    } else {
      sched_ok = sched;
    }
    tm.sync();
  }
  if (misc[0]) {  // dof_entries / dof_depth of the tree are smaller than its DOF tree: refuse
    for (int i = tl; i < nq; i += T) P.r.x[qoff + i] = P.b.x0[qoff + i];
    if (tl == 0) {
      P.r.iters[prob] = 0;
      P.r.status[prob] = BR_IK_MAXITER | (BR_IK_FLAG_BADTREE << 8);
      P.r.cost[prob] = __int_as_float(0x7fc00000);  // NaN
    }
    tm.sync();
    return;
  }
  const int nL = rowoff[nv];
  // ascending list of the tangent columns that move each target frame (its support)
  for (int t = 0; t < nt; ++t) {
    const unsigned long long sp = support[fparent[t]];
    int base = 0;
#pragma unroll 1
    for (int c0 = 0; c0 < nv; c0 += T) {
      const int c = c0 + tl;
      const bool in = c < nv && ((sp >> cjoint[c]) & 1ull);
      const unsigned bal = (__ballot_sync(tm.mask, in) >> ((threadIdx.x & 31) - tl)) &
                           (T == 32 ? 0xffffffffu : ((1u << T) - 1u));
      if (in) sup[t * nv + base + __popc(bal & ((1u << tl) - 1u))] = (unsigned char)c;
      base += __popc(bal);
    }
    if (tl == 0) nsup[t] = base;
  }
  tm.sync();

  // ---- helpers ------------------------------------------------------------
  // float64 FK of configuration q (shared) -> world poses (returned buffer), pointer jumping.
  auto fk = [&](const double* q) -> double* {
    for (int j = tl; j < nj; j += T) {
      const DPose Lj = dlocal_transform<kGeneral>(jtype[j], to_d(ld8(place + 8 * j)), axis + 4 * j, q + idxq[j]);
      sts(poseA, nj, j, Lj);
      ancA[j] = parent[j];
    }
    tm.sync();
    double* A = poseA;
    double* B = poseB;
    int* aA = ancA;
    int* aB = ancB;
    for (int r = 0; r < tree.rounds; ++r) {
      for (int j = tl; j < nj; j += T) {
        const int a = aA[j];
        if (a >= 0) {
          sts(B, nj, j, dcompose(lds(A, nj, a), lds(A, nj, j)));
          aB[j] = aA[a];
        } else {
          sts(B, nj, j, lds(A, nj, j));
          aB[j] = -1;
        }
      }
      tm.sync();
      double* tp = A; A = B; B = tp;
      int* ta = aA; aA = aB; aB = ta;
    }
    return A;
  };

  // float64 residual of the stack at q with world poses `pose`: fills tw, xi, dr; returns 0.5 |r|^2.
  // the parent joint of this lane's first target, read once: the residual's first pose load
  // then follows FK's last barrier directly
  const int fpar_own = tl < nt ? fparent[tl] : 0;
  auto residual = [&](const double* q, const double* pose) -> double {
    double acc = 0.0;
    // one pass over the targets (jobs 0..nt-1) and, for the rest term, the joints (jobs
    // nt..nt+nj-1), so that the SE3 log of pose targets and free-flyer rest residuals has
    // one call site
    const int njobs = nt + (use_rest ? nj : 0);
    for (int jb = tl; jb < njobs; jb += T) {
      DPose rel;
      double* out = nullptr;  // 6 slots [v, w] when rel's SE3 log is wanted
      double wv = 0.0, ww = 0.0;
      if (jb < nt) {
        const int t = jb;
        const DPose Tee = dcompose(lds(pose, nj, jb < T ? fpar_own : fparent[t]), to_d(ld8(fplace + 8 * t)));
        std8(tw + 8 * t, Tee);
        double* e = xi + 8 * t;
        const DPose Tt = ldd(tgt + 8 * t);
        const int kind = kGeneral ? tkind[t] : BR_TARGET_POSE;
        if (kind == BR_TARGET_POSITION) {                            // pose.py:127-131
          const double3 dp = dsub(Tee.t, Tt.t);
          e[0] = dp.x; e[1] = dp.y; e[2] = dp.z; e[3] = 0.0; e[4] = 0.0; e[5] = 0.0;
          acc += wpd * wpd * ddot(dp, dp);
        } else if (kind == BR_TARGET_ORIENTATION) {                  // pose.py:165-173
          const double3 w = dso3_log(dqmul(dqconj(Tt.q), Tee.q));
          e[0] = 0.0; e[1] = 0.0; e[2] = 0.0; e[3] = w.x; e[4] = w.y; e[5] = w.z;
          acc += wod * wod * ddot(w, w);
        } else {
          rel = dcompose(dinverse(Tt), Tee);                         // pose.py:63-64
          out = e;
          wv = wpd;
          ww = wod;
        }
      } else {                                                       // regularization.py:48-54
        const int j = jb - nt;
        const int jt = jtype[j];
        const int iq = idxq[j], iv = idxv[j];
        if (kGeneral ? joint_is_vector(jt) : (jt == BR_JOINT_REVOLUTE || jt == BR_JOINT_PRISMATIC)) {
          for (int k = 0; k < (kGeneral ? joint_nv(jt) : 1); ++k) {
            const double dd = q[iq + k] - qrest[iq + k];
            dr[iv + k] = dd;
            acc += wrd * wrd * dd * dd;
          }
        } else if (kGeneral && jt == BR_JOINT_SPHERICAL) {           // spherical.py:58-62
          const double3 w = dso3_log(dqnormalize(dqmul(
              dqconj(make_double4(qrest[iq], qrest[iq + 1], qrest[iq + 2], qrest[iq + 3])),
              make_double4(q[iq], q[iq + 1], q[iq + 2], q[iq + 3]))));
          dr[iv] = w.x; dr[iv + 1] = w.y; dr[iv + 2] = w.z;
          acc += wrd * wrd * ddot(w, w);
        } else if (kGeneral && (jt == BR_JOINT_PLANAR || jt == BR_JOINT_REVOLUTE_UNBOUNDED)) {  // planar.py:70-76, revolute.py:233-237
          const int k = jt == BR_JOINT_PLANAR ? 2 : 0;
          const double dth = atan2(q[iq + k + 1], q[iq + k]) - atan2(qrest[iq + k + 1], qrest[iq + k]);
          if (jt == BR_JOINT_PLANAR) {
            const double dx = q[iq] - qrest[iq], dy = q[iq + 1] - qrest[iq + 1];
            dr[iv] = dx; dr[iv + 1] = dy; dr[iv + 2] = dth;
            acc += wrd * wrd * (dx * dx + dy * dy + dth * dth);
          } else {
            dr[iv] = dth;
            acc += wrd * wrd * dth * dth;
          }
        } else if (jt == BR_JOINT_FREE_FLYER) {                      // free_flyer.py:53-57
          const DPose a{d3(qrest[iq], qrest[iq + 1], qrest[iq + 2]),
                        make_double4(qrest[iq + 3], qrest[iq + 4], qrest[iq + 5], qrest[iq + 6])};
          const DPose b{d3(q[iq], q[iq + 1], q[iq + 2]), make_double4(q[iq + 3], q[iq + 4], q[iq + 5], q[iq + 6])};
          rel = dcompose(dinverse(a), b);
          out = dr + iv;
          wv = wrd;
          ww = wrd;
        }
      }
      if (out) {
        double3 v, w;
        dse3_log(rel, v, w);
        out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = w.x; out[4] = w.y; out[5] = w.z;
        acc += wv * wv * ddot(v, v) + ww * ww * ddot(w, w);
      }
    }
    if (use_limits) {                                                // limits.py:56-62
#pragma unroll 1
      for (int i = tl; i < nq; i += T) {
        const double lo = fmax((double)lower[i] - q[i], 0.0), hi = fmax(q[i] - (double)upper[i], 0.0);
        acc += wld * wld * (lo * lo + hi * hi);
      }
    }
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(tm.mask, acc, o, T);
    tm.sync();
    return 0.5 * acc;
  };

  // float32 J^T J (packed lower, column-major) and g = J^T r at q with world poses `pose`; returns |g|.
  // Each target's pose Jacobian diag(w) Jr^-1 blockdiag(R^T, R^T) J_lwa (pose.py:68-103) is
  // built only on its support columns and accumulated into the (support x support) block.
  auto build_normal = [&](const double* q, const double* pose) -> R {
    for (int c = tl; c < nv; c += T) {
      if constexpr (kF64) {
        const DPose Tj = lds(pose, nj, cjoint[c]);
        const double3 a = dqrot(Tj.q, d3(caxis[4 * c], caxis[4 * c + 1], caxis[4 * c + 2]));
        double* cw = colw + 8 * c;
        cw[0] = a.x; cw[1] = a.y; cw[2] = a.z; cw[4] = Tj.t.x; cw[5] = Tj.t.y; cw[6] = Tj.t.z;
      } else {
        const Pose Tj = to_f(lds(pose, nj, cjoint[c]));
        const float3 a = qrot(Tj.q, f3(caxis[4 * c], caxis[4 * c + 1], caxis[4 * c + 2]));
        *reinterpret_cast<float4*>(colw + 8 * c) = make_float4(a.x, a.y, a.z, 0.f);
        *reinterpret_cast<float4*>(colw + 8 * c + 4) = make_float4(Tj.t.x, Tj.t.y, Tj.t.z, 0.f);
      }
      g[c] = (R)0;
    }
    // Jr^-1 of each target: its three B columns on three lanes (job = 3 t + c)
    for (int job = tl; job < 3 * nt; job += T) {
      const int t = job / 3, c = job - 3 * t;
      const double* e = xi + 8 * t;
      R* o = jri + 16 * t;
      if (!kGeneral || tkind[t] == BR_TARGET_POSE) {                   // SE3 Jr^-1(xi), tangents.py:204-207
        if constexpr (kF64) {
          double b0, b1, b2;
          const double3 bc = djr_inv_se3_col<9>(d3(e[0], e[1], e[2]), d3(e[3], e[4], e[5]), c, b0, b1, b2);
          if (c == 0) { o[0] = e[3]; o[1] = e[4]; o[2] = e[5]; o[3] = b0; o[4] = b1; o[5] = b2; }
          o[6 + c] = bc.x; o[9 + c] = bc.y; o[12 + c] = bc.z;
        } else {
          float b0, b1, b2;
          const float3 w = f3((float)e[3], (float)e[4], (float)e[5]);
          const float3 bc = jr_inv_se3_col<9>(f3((float)e[0], (float)e[1], (float)e[2]), w, c, b0, b1, b2);
          if (c == 0) { o[0] = w.x; o[1] = w.y; o[2] = w.z; o[3] = b0; o[4] = b1; o[5] = b2; }
          o[6 + c] = bc.x; o[9 + c] = bc.y; o[12 + c] = bc.z;
        }
      } else if (c == 0) {  // orientation: SO3 Jr^-1(r) (tangents.py:122-145) as the angular block, no coupling;
                            // position: identity (its rows are replaced by J_lwa's linear rows)
        const bool ori = tkind[t] == BR_TARGET_ORIENTATION;
        o[0] = (R)e[3]; o[1] = (R)e[4]; o[2] = (R)e[5];
        o[3] = (R)1;
        o[4] = ori ? (R)0.5 : (R)0;
        if constexpr (kF64) {
          o[5] = ori ? dvinv_coeff(e[3] * e[3] + e[4] * e[4] + e[5] * e[5]) : 0.0;
        } else {
          const float3 w = f3((float)e[3], (float)e[4], (float)e[5]);
          o[5] = ori ? vinv_coeff(dot(w, w)) : 0.f;
        }
        for (int k = 0; k < 9; ++k) o[6 + k] = (R)0;
      }
    }
#pragma unroll 1
    for (int e = tl; e < nL; e += T) jtj[e] = (R)0;
    tm.sync();
    // Jacobian columns of two targets per pass (blocks Jc_h = work + 6 nv h, h = 0, 1: row r of
    // target t0 + h's J on its support columns), then each target's J^T J and J^T r in target
    // order, so the accumulation order (and rounding) does not depend on the pairing
    for (int t0 = 0; t0 < nt; t0 += 2) {
      const int npair = t0 + 1 < nt ? 2 : 1;
      const int ns0 = nsup[t0];
      const int njob = ns0 + (npair == 2 ? nsup[t0 + 1] : 0);
      for (int job = tl; job < njob; job += T) {
        const int h = job >= ns0 ? 1 : 0;
        const int t = t0 + h, u = job - (h ? ns0 : 0);
        const int kind = kGeneral ? tkind[t] : BR_TARGET_POSE;
        const int c = sup[t * nv + u];
        R* Jc = work + 6 * nv * h;
        if constexpr (kF64) {
          const DPose Tee = ldd(tw + 8 * t);
          const double* o = jri + 16 * t;
          DJrInv J;
          J.w = d3(o[0], o[1], o[2]);
          J.b0 = o[3]; J.b1 = o[4]; J.b2 = o[5];
#pragma unroll
          for (int k = 0; k < 9; ++k) J.B[k] = o[6 + k];
          const double4 qc = dqconj(Tee.q);
          const double* cw = colw + 8 * c;
          const double3 a = d3(cw[0], cw[1], cw[2]);
          double3 lin, ang;
          if (ckind[c] == 0) {
            lin = dcross(a, dsub(Tee.t, d3(cw[4], cw[5], cw[6])));      // jacobian.py:213-215
            ang = a;
          } else {
            lin = a;
            ang = d3(0.0, 0.0, 0.0);
          }
          double3 ol, oa;
          djr_inv_apply(J, dqrot(qc, lin), dqrot(qc, ang), ol, oa);    // pose.py:91-99
          if (kind == BR_TARGET_POSITION) {            // top rows of J_lwa (pose.py:133-141)
            ol = lin;
            oa = d3(0.0, 0.0, 0.0);
          } else if (kind == BR_TARGET_ORIENTATION) {  // Jr^-1(r) R^T J_ang (pose.py:175-195)
            ol = d3(0.0, 0.0, 0.0);
          }
          Jc[u] = wp * ol.x; Jc[nv + u] = wp * ol.y; Jc[2 * nv + u] = wp * ol.z;
          Jc[3 * nv + u] = wo * oa.x; Jc[4 * nv + u] = wo * oa.y; Jc[5 * nv + u] = wo * oa.z;
        } else {
          const Pose Tee = to_f(ldd(tw + 8 * t));
          const float* o = jri + 16 * t;
          JrInv J;
          J.w = f3(o[0], o[1], o[2]);
          J.b0 = o[3]; J.b1 = o[4]; J.b2 = o[5];
#pragma unroll
          for (int k = 0; k < 9; ++k) J.B[k] = o[6 + k];
          const float4 a4 = *reinterpret_cast<const float4*>(colw + 8 * c);
          const float3 a = f3(a4.x, a4.y, a4.z);
          float3 lin, ang;
          if (ckind[c] == 0) {
            const float4 o4 = *reinterpret_cast<const float4*>(colw + 8 * c + 4);
            lin = cross(a, sub(Tee.t, f3(o4.x, o4.y, o4.z)));             // jacobian.py:213-215
            ang = a;
          } else {
            lin = a;
            ang = f3(0.f, 0.f, 0.f);
          }
          float3 ol, oa;
          jr_inv_apply(J, qrot_inv(Tee.q, lin), qrot_inv(Tee.q, ang), ol, oa);  // pose.py:91-99
          if (kind == BR_TARGET_POSITION) {            // top rows of J_lwa (pose.py:133-141)
            ol = lin;
            oa = f3(0.f, 0.f, 0.f);
          } else if (kind == BR_TARGET_ORIENTATION) {  // Jr^-1(r) R^T J_ang (pose.py:175-195)
            ol = f3(0.f, 0.f, 0.f);
          }
          Jc[u] = wp * ol.x; Jc[nv + u] = wp * ol.y; Jc[2 * nv + u] = wp * ol.z;
          Jc[3 * nv + u] = wo * oa.x; Jc[4 * nv + u] = wo * oa.y; Jc[5 * nv + u] = wo * oa.z;
        }
      }
      tm.sync();
      for (int h = 0; h < npair; ++h) {
      const int t = t0 + h;
      const int ns = nsup[t];
      const unsigned char* st = sup + t * nv;
      const R* Jc = work + 6 * nv * h;
      const double* e = xi + 8 * t;
      R kw[6] = {(R)1, (R)1, (R)1, (R)1, (R)1, (R)1};  // IRLS weight of each of the target's 6 rows
      if (irls) {
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          const double rr = (r < 3 ? wpd : wod) * e[r];
          kw[r] = irls_weight<R>(S.kernel, kc, rr * rr);
        }
      }
      for (int p = tl; p < tri(ns); p += T) {
        const int uv = decode_pair(p);                        // row-major (u >= v) decode of p
        const int u = uv & 0xff, v = uv >> 8;
        R acc = (R)0;
        if (irls) {
#pragma unroll
          for (int r = 0; r < 6; ++r) acc = rfma(Jc[r * nv + u] * kw[r], Jc[r * nv + v], acc);
        } else {
#pragma unroll
          for (int r = 0; r < 6; ++r) acc = rfma(Jc[r * nv + u], Jc[r * nv + v], acc);
        }
        jtj[rowoff[st[u]] + ddep[st[v]]] += acc;  // st ascending: st[u] descends from st[v]
      }
      const R rw[6] = {wp * (R)e[0] * kw[0], wp * (R)e[1] * kw[1], wp * (R)e[2] * kw[2],
                       wo * (R)e[3] * kw[3], wo * (R)e[4] * kw[4], wo * (R)e[5] * kw[5]};
      for (int u = tl; u < ns; u += T) {
        R acc = (R)0;
#pragma unroll
        for (int r = 0; r < 6; ++r) acc = rfma(Jc[r * nv + u], rw[r], acc);
        g[st[u]] += acc;
      }
      tm.sync();
      }
    }
    // rest (w I, regularization.py:56-64) and limit (+-w on active rows, limits.py:64-86) terms
    R gg = (R)0;
    for (int c = tl; c < nv; c += T) {
      R dg = (R)0, gc = g[c];
      if (use_rest) {
        const double rr = wrd * dr[c];
        const R w = irls ? irls_weight<R>(S.kernel, kc, rr * rr) : (R)1;
        dg += wr * wr * w;
        gc += wr * wr * w * (R)dr[c];
      }
      if (use_limits) {
        const int j = cjoint[c];
        if (joint_is_vector(jtype[j])) {  // nq == nv: +-w on active rows; other kinds give zero rows (limits.py:42-54)
          const int iq = idxq[j] + (c - idxv[j]);
          if (q[iq] < (double)lower[iq]) {
            const double d = (double)lower[iq] - q[iq];
            const R w = irls ? irls_weight<R>(S.kernel, kc, wld * wld * d * d) : (R)1;
            dg += wl * wl * w;
            gc -= wl * wl * w * (R)d;
          }
          if (q[iq] > (double)upper[iq]) {
            const double d = q[iq] - (double)upper[iq];
            const R w = irls ? irls_weight<R>(S.kernel, kc, wld * wld * d * d) : (R)1;
            dg += wl * wl * w;
            gc += wl * wl * w * (R)d;
          }
        }
      }
      jtj[rowoff[c] + ddep[c]] += dg;
      g[c] = gc;
      gg += gc * gc;
    }
#pragma unroll
    for (int o = T / 2; o > 0; o >>= 1) gg += __shfl_xor_sync(tm.mask, gg, o, T);
    tm.sync();
    return rsqrt_(gg);
  };

  // Solve (J^T J + damp I) delta = -g in float32 by an LDL^T factorization that eliminates
  // the DOF tree leaves first (Featherstone's LTL order: no fill-in).  Eliminating DOF k
  // updates only pairs of its ancestors, A_ij -= A_ki A_kj / d_k, lanes over those pairs,
  // one team sync per DOF; entries stay unscaled (A_ki = l_ik d_k) and the damping is
  // added to each pivot as it is read.  d_k > 0 for every k is the test a Cholesky
  // factorization applies.  The triangular solves run in registers (lane tl owns DOFs
  // tl + T r), one shuffle per step.  Returns false if a pivot is not positive and finite.
  // Level-scheduled factorization: the DOFs of one height in the DOF tree are
  // eliminated together (tasks of the schedule, one lane each), the right-hand side
  // -g is updated in the same tasks (forward substitution), then back substitution
  // runs root first by depth: delta_i = (z_i - sum_a Lm[i][a] delta_anc(i, a)) / D_i.
  auto solve = [&](R damp) -> bool {
    R* Lm = work;
    R* z = work + nL;
    {  // Lm = J^T J, 16-byte vectors (both regions start on a 16-byte boundary)
      using V = typename std::conditional<kF64, double2, float4>::type;
      constexpr int VW = 16 / (int)sizeof(R);
      const int nvec = nL / VW;
#pragma unroll 1
      for (int e = tl; e < nvec; e += T) reinterpret_cast<V*>(Lm)[e] = reinterpret_cast<const V*>(jtj)[e];
      for (int e = nvec * VW + tl; e < nL; e += T) Lm[e] = jtj[e];
    }
    // pivots of the leaves (final already); a non-leaf's is stored by the task that
    // finalises its diagonal (the schedule's flag).  A pivot is tested where it becomes
    // final: in its flagged task for a non-leaf, and here for every DOF (while the pivots
    // below a non-leaf are positive its pivot only decreases from this value, so the test
    // here fails for it only when the final one would: the outcome of one test at the end).
    bool bad = false;
    for (int i = tl; i < nv; i += T) {
      z[i] = -g[i];
      const R piv = jtj[rowoff[i] + ddep[i]] + damp;
      bad |= !(piv > (R)0) || !isfinite(piv);
      dinv[i] = rrcp(piv);
    }
    tm.sync();
    const int nlev = (int)sched[0];
    const int toff = (5 + nlev + 3) & ~3;
    const uint4* tasks = reinterpret_cast<const uint4*>(sched + toff);
    const uint2* extra = reinterpret_cast<const uint2*>(sched + toff + 4 * (int)sched[1]);
    // this lane's first task of level l + 1 is loaded during level l (its index clamped to the
    // last task, used only when it lies in level l + 1)
    const int last = (int)sched[1] - 1;
    int t0 = 0;
    uint4 first = last >= 0 ? __ldg(tasks + (tl < last ? tl : last)) : make_uint4(0u, 0u, 0u, 0u);
    // the trunk's levels run in registers in the float64 variants only (measured on the
    // 8,192-problem mix: float64 4.05 -> 4.00 ms, float32 2.76 -> 2.80 ms, outcomes identical)
    const int ntr = kF64 ? misc[2] : 0;
    for (int l = 0; l < nlev - ntr; ++l) {
      const int t1 = (int)__ldg(sched + 5 + l);
      int p = t0 + tl;
      uint4 nx = p < t1 ? first : make_uint4(0u, 0u, 0u, 0u);
      if (last >= 0) first = __ldg(tasks + (t1 + tl < last ? t1 + tl : last));
      t0 = t1;
      for (; p < t1; p += T) {
        const uint4 tk = nx;                                   // the next pass's task is in flight
        if (p + T < t1) nx = __ldg(tasks + p + T);
        const int dst = tk.x & 0xffff;
        R acc = rfma(-Lm[tk.y & 0xffff] * dinv[tk.z & 0xffff], Lm[tk.y >> 16], Lm[dst]);
        int e = (int)(tk.z >> 16);
        const int e1 = e + (int)(tk.x >> 16);
        for (; e + 1 < e1; e += 2) {                           // two records in flight at once
          const uint2 ea = __ldg(extra + e), eb = __ldg(extra + e + 1);
          const R a1 = Lm[ea.x & 0xffff] * dinv[ea.y], a2 = Lm[ea.x >> 16];
          const R b1 = Lm[eb.x & 0xffff] * dinv[eb.y], b2 = Lm[eb.x >> 16];
          acc = rfma(-a1, a2, acc);
          acc = rfma(-b1, b2, acc);
        }
        if (e < e1) {
          const uint2 ex = __ldg(extra + e);
          acc = rfma(-Lm[ex.x & 0xffff] * dinv[ex.y], Lm[ex.x >> 16], acc);
        }
        Lm[dst] = acc;
        if (tk.w) {                                            // DOF tk.w - 1's pivot is final
          const R piv = acc + damp;
          bad |= !(piv > (R)0) || !isfinite(piv);
          dinv[tk.w - 1] = rrcp(piv);
        }
      }
      tm.sync();
    }
    if (ntr > 0) {
      // The trunk's levels in registers: lane t < ne holds the trunk's factor entry t (row i,
      // column j at t = i (i + 1) / 2 + j: the trunk rows are the first entries of the factor),
      // lane ne + i the right-hand side z_i; each elimination takes its operands by shuffles
      // instead of a pass over shared memory and a team synchronisation.  The same operations
      // in the same order as the schedule's tasks of those levels (one contribution per entry
      // and level), so the factor is the same to the bit.
      const int ne = ntr * (ntr + 1) / 2;
      const bool ent = tl < ne, rhs = !ent && tl < ne + ntr;
      int ri = 0, cj = 0;
      if (ent) {
#pragma unroll 1
        while (tri(ri + 1) <= tl) ++ri;
        cj = tl - tri(ri);
      } else if (rhs) {
        ri = tl - ne;
      }
      R v = ent ? Lm[tl] : rhs ? z[ri] : (R)0;
      R dk = dinv[ntr - 1];                                    // final since the levels below
#pragma unroll 1
      for (int k = ntr - 1; k >= 1; --k) {                     // eliminate DOF k
        const int rk = tri(k);
        const R lki = __shfl_sync(tm.mask, v, rk + (ri < k ? ri : 0));
        const R lkj = __shfl_sync(tm.mask, v, ent ? rk + (cj < k ? cj : 0) : ne + k);
        if ((ent || rhs) && ri < k) v = rfma(-lki * dk, lkj, v);
        const R piv = __shfl_sync(tm.mask, v, tri(k - 1) + k - 1) + damp;   // DOF k - 1's, final
        bad |= !(piv > (R)0) || !isfinite(piv);
        dk = rrcp(piv);
        if (tl == 0) dinv[k - 1] = dk;
      }
      if (ent) Lm[tl] = v;
      else if (rhs) z[ri] = v;
      tm.sync();
    }
    if (__any_sync(tm.mask, bad)) return false;
    // back substitution by depth, root first: a lane keeps its DOFs' right-hand sides in
    // registers; once the DOFs of depth dl are final, every deeper DOF subtracts the
    // term of its one ancestor at depth dl (no two lanes write the same DOF)
    constexpr int NR = lm_rows(T);
    R zr[NR], dvr[NR];
    int dr[NR], ror[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const int i = tl + T * r;
      const bool in = i < nv;
      zr[r] = in ? z[i] : (R)0;
      dvr[r] = in ? dinv[i] : (R)0;
      dr[r] = in ? ddep[i] : -1;
      ror[r] = in ? rowoff[i] : 0;
    }
    const int ndl = misc[1];
#pragma unroll 1
    for (int dl = 0; dl < ndl; ++dl) {
      // this depth's factor entries and ancestors do not depend on the synchronisation below:
      // loaded before it, so that only the ancestor's delta is read after it
      R lf[NR];
      int an[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const bool deeper = dr[r] > dl;
        lf[r] = deeper ? Lm[ror[r] + dl] : (R)0;
        an[r] = deeper ? ancd[(tl + T * r) * L.anc_stride + dl] : 0;
      }
#pragma unroll
      for (int r = 0; r < NR; ++r)
        if (dr[r] == dl) delta[tl + T * r] = zr[r] * dvr[r];
      tm.sync();
#pragma unroll
      for (int r = 0; r < NR; ++r)
        if (dr[r] > dl) zr[r] = rfma(-lf[r], delta[an[r]], zr[r]);
    }
    tm.sync();
    return true;
  };

  // x_new = clamp(integrate(x, delta)) in float64
  auto retract = [&]() {
    for (int j = tl; j < nj; j += T) {
      const int jt = jtype[j];
      const int iq = idxq[j], iv = idxv[j];
      auto clampq = [&](int k, double v) { xn[iq + k] = fmin(fmax(v, (double)lower[iq + k]), (double)upper[iq + k]); };
      if (kGeneral ? joint_is_vector(jt) : (jt == BR_JOINT_REVOLUTE || jt == BR_JOINT_PRISMATIC)) {
        for (int k = 0; k < (kGeneral ? joint_nv(jt) : 1); ++k) clampq(k, x[iq + k] + (double)delta[iv + k]);
      } else if (kGeneral && jt == BR_JOINT_SPHERICAL) {             // spherical.py:52-56
        const double4 n = dqnormalize(dqmul(make_double4(x[iq], x[iq + 1], x[iq + 2], x[iq + 3]),
                                            dse3_exp(d3(0.0, 0.0, 0.0), d3(delta[iv], delta[iv + 1], delta[iv + 2])).q));
        clampq(0, n.x); clampq(1, n.y); clampq(2, n.z); clampq(3, n.w);
      } else if (kGeneral && (jt == BR_JOINT_PLANAR || jt == BR_JOINT_REVOLUTE_UNBOUNDED)) {  // planar.py:61-68, revolute.py:223-231
        const int k = jt == BR_JOINT_PLANAR ? 2 : 0;
        const double th = atan2(x[iq + k + 1], x[iq + k]) + (double)delta[iv + k];
        double s, c;
        sincos(th, &s, &c);
        if (jt == BR_JOINT_PLANAR) {
          clampq(0, x[iq] + (double)delta[iv]);
          clampq(1, x[iq + 1] + (double)delta[iv + 1]);
        }
        clampq(k, c);
        clampq(k + 1, s);
      } else if (jt == BR_JOINT_FREE_FLYER) {                        // free_flyer.py:47-51
        // plain variant: the float32 step's exponential in float32 (its rounding is relative
        // to the step), composed with the float64 iterate in float64; the general variant
        // keeps the float64 exponential
        const DPose a{d3(x[iq], x[iq + 1], x[iq + 2]), make_double4(x[iq + 3], x[iq + 4], x[iq + 5], x[iq + 6])};
        DPose inc;
        if (kGeneral || kF64) {
          inc = dse3_exp(d3(delta[iv], delta[iv + 1], delta[iv + 2]), d3(delta[iv + 3], delta[iv + 4], delta[iv + 5]));
        } else {
          const Pose e = se3_exp_step(f3((float)delta[iv], (float)delta[iv + 1], (float)delta[iv + 2]),
                                      f3((float)delta[iv + 3], (float)delta[iv + 4], (float)delta[iv + 5]));
          inc = DPose{d3(e.t.x, e.t.y, e.t.z), make_double4(e.q.x, e.q.y, e.q.z, e.q.w)};
        }
        DPose n = dcompose(a, inc);
        n.q = dqnormalize(n.q);
        xn[iq] = n.t.x; xn[iq + 1] = n.t.y; xn[iq + 2] = n.t.z;
        xn[iq + 3] = n.q.x; xn[iq + 4] = n.q.y; xn[iq + 5] = n.q.z; xn[iq + 6] = n.q.w;
#pragma unroll 1
        for (int k = 0; k < 7; ++k) clampq(k, xn[iq + k]);
      }
    }
    tm.sync();
  };

  // ---- the LM / GN loop (levenberg_marquardt.py:83-135, gauss_newton.py:27-76) ----
  // fk, residual and solve each have ONE call site (they are inlined lambdas: a second
  // site would duplicate their code and the kernel's instruction footprint): the first
  // pass evaluates the start, every later pass the trial point of one iteration, and a
  // last pass re-evaluates x when the stacked residual is wanted and the final trial
  // point was rejected.
  const bool gn = S.optimizer == BR_OPT_GN;
  const bool want_residual = P.r.residual && P.b.r_offset;
  R lam = gn ? (R)0 : (R)S.lam0;
  R gnorm = (R)0;
  double cost = 0.0;
  bool need_jac = true, started = false, final_pass = false, last_at_x = true;
  int flags = 0;
  int status = BR_IK_MAXITER;
  int it = 0;
  const double* xe = x;  // the point the next pass evaluates
  for (;;) {
    double* pose = fk(xe);
    const double cn = residual(xe, pose);
    if (final_pass) break;
    if (!started) {
      started = true;
      cost = cn;
      flags = isfinite(cost) ? 0 : BR_IK_FLAG_NONFINITE;
    } else {
      ++it;
      if (!isfinite(cn)) flags |= BR_IK_FLAG_NONFINITE;
      if (gn || cn < cost) {
#pragma unroll 1
        for (int i = tl; i < nq; i += T) x[i] = xn[i];
        tm.sync();
        cost = cn;
        if (!gn) lam = rmax(lam / (R)S.factor, (R)S.lam_min);
        need_jac = true;
        last_at_x = true;
        if (gnorm < (R)S.tol) { status = BR_IK_CONVERGED; break; }
      } else {
        lam = rmin(lam * (R)S.factor, (R)S.lam_max);
        last_at_x = false;
      }
    }
    if (it >= S.max_iter) {
      if (want_residual && !last_at_x) {
        final_pass = true;
        xe = x;
        continue;
      }
      break;
    }
    if (need_jac) {  // pose holds FK(x) here: x was the last point evaluated and kept
      gnorm = build_normal(x, pose);
      need_jac = false;
    }
    const R damp = gn ? (R)S.gn_eps : lam;
    // a failed factorization is retried with diagonal regularisation 1e-6 .. 1e-1
    bool ok = false;
    R extra = (R)0;
    for (int k = 0; k < 7; ++k) {
      ok = solve(damp + extra);
      if (ok) break;
      flags |= BR_IK_FLAG_REGULARIZED;
      extra = k == 0 ? (R)1e-6f : extra * (R)10;
    }
    if (!ok) {
#pragma unroll 1
      for (int i = tl; i < nv; i += T) delta[i] = (R)0;
      tm.sync();
    }
    retract();
    xe = xn;
  }
  // ---- results ------------------------------------------------------------
#pragma unroll 1
  for (int i = tl; i < nq; i += T) P.r.x[qoff + i] = (float)x[i];
  if (want_residual) {
    // stacked residual at the returned x, CostStack order (stack.py:104-117); the residual
    // buffers hold x's values (last pass above)
    float* out = P.r.residual + P.b.r_offset[prob];
    int o = 0;  // rows of the targets: 6 per pose, 3 per position or orientation target
#pragma unroll 1
    for (int t = 0; t < nt; ++t) {
      const double* e = xi + 8 * t;
      const int kind = kGeneral ? tkind[t] : BR_TARGET_POSE;
      if (tl == 0) {
        if (kind != BR_TARGET_ORIENTATION) {
          out[o + 0] = (float)(wpd * e[0]); out[o + 1] = (float)(wpd * e[1]); out[o + 2] = (float)(wpd * e[2]);
        }
        if (kind != BR_TARGET_POSITION) {
          const int a = kind == BR_TARGET_POSE ? o + 3 : o;
          out[a + 0] = (float)(wod * e[3]); out[a + 1] = (float)(wod * e[4]); out[a + 2] = (float)(wod * e[5]);
        }
      }
      o += kind == BR_TARGET_POSE ? 6 : 3;
    }
    if (use_limits) {  // the limit and rest rows keep their place when their weight is 0
#pragma unroll 1
      for (int i = tl; i < nq; i += T) {
        out[o + i] = (float)(wld * fmax((double)lower[i] - x[i], 0.0));
        out[o + nq + i] = (float)(wld * fmax(x[i] - (double)upper[i], 0.0));
      }
    }
    o += 2 * nq;
    if (use_rest)
#pragma unroll 1
      for (int c = tl; c < nv; c += T) out[o + c] = (float)(wrd * dr[c]);
  }
  if (tl == 0) {
    P.r.iters[prob] = it;
    P.r.status[prob] = status | (flags << 8);
    P.r.cost[prob] = (float)cost;
  }
  tm.sync();
}

template <int T, bool kGeneral, bool kF64>
__device__ __forceinline__ void run_item(const LmParams& P, int cls, int first, int count, float* wsm, int lane,
                                         const uint32_t*& sched_ok) {
  const int team = lane / T;
  Team<T> tm;
  tm.tl = lane % T;
  tm.mask = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (team * T));
  const br_tree_t& tree = P.trees[cls];
  const TeamLayout L(tree.njoints, tree.nq, tree.nv, P.b.max_targets, T, tree.dof_entries, tree.dof_depth, tree.rounds,
                     kF64 ? 2 : 1);
  if (team < count) {
    const int prob = P.b.order[first + team];
    solve_problem<T, kGeneral, kF64>(P, tree, prob, wsm + team * L.total, tm, sched_ok);
  }
}

template <bool kGeneral, bool kF64>
__global__ void __maxnreg__(kF64 ? 168 : 128) lm_solve_kernel(const LmParams P) {
  extern __shared__ __align__(16) float smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float* wsm = smem + (size_t)warp * P.warp_floats;
  const uint32_t* sched_ok = nullptr;  // the level schedule this team has checked
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(P.queue, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= P.b.n_items) break;
    const int first = P.b.items[3 * item], count = P.b.items[3 * item + 1], cls = P.b.items[3 * item + 2];
    // One instantiation: 32-lane teams.  8- and 16-lane teams (several small problems per
    // warp) were measured slower on the mixed batch: three copies of this kernel body
    // overflow the instruction cache, and 32 lanes are the fastest per class on their own.
    run_item<kLmTeam, kGeneral, kF64>(P, cls, first, count, wsm, lane, sched_ok);
    __syncwarp();
  }
}

}  // namespace br

using namespace br;

extern "C" int64_t br_lm_team_floats(const br_tree_t* tree, int32_t max_targets) {
  if (!tree || max_targets < 0) return BR_EINVAL;
  const int T = kLmTeam;
  return TeamLayout(tree->njoints, tree->nq, tree->nv, max_targets, T, tree->dof_entries, tree->dof_depth, tree->rounds).total;
}

#include <mutex>

namespace {
std::mutex g_lm_mu;  // guards the two per-device caches below
// Dynamic shared memory each lm_solve_kernel variant has been allowed on each device
// (cudaFuncAttributeMaxDynamicSharedMemorySize only ever raised, so a launch that
// needs less than an earlier one still fits).  Shared by every entry point below.
int g_smem_allowed[4][64] = {};  // [float64 variant * 2 + general variant][device]
}  // namespace

// Argument checks of both LM entry points: BR_OK, an error, or kLmNothing when the batch
// has no problem to launch.
constexpr int kLmNothing = 1;
static int lm_check(const br_ik_batch_t* batch, const br_ik_settings_t* settings, const br_ik_result_t* result,
                    int32_t warps_per_cta) {
  if (!batch || !settings || !result) return BR_EINVAL;
  const br_ik_batch_t& b = *batch;
  if (b.n_problems < 0 || b.n_items < 0 || b.n_classes < 1) return BR_EINVAL;
  if (b.n_classes > BR_MAX_IK_CLASSES || b.max_targets > BR_MAX_IK_TARGETS) return BR_ETOOBIG;
  if (b.max_targets < 1 || !b.trees || !b.team_size) return BR_EINVAL;
  if (b.n_problems == 0 || b.n_items == 0) return kLmNothing;
  if (!b.items || !b.order || !b.n_targets || !b.frames || !b.targets || !b.q_offset || !b.x0 || !b.q_rest)
    return BR_EINVAL;
  if (!result->x || !result->iters || !result->status || !result->cost) return BR_EINVAL;
  if (settings->max_iter < 0) return BR_EINVAL;
  if (settings->kernel < BR_KERNEL_L2 || settings->kernel > BR_KERNEL_TUKEY) return BR_EINVAL;
  if (settings->kernel != BR_KERNEL_L2 && !(settings->kernel_param > 0.f)) return BR_EINVAL;
  if (warps_per_cta < 1 || warps_per_cta > 32) return BR_EINVAL;
  if (settings->precision != BR_PREC_F32 && settings->precision != BR_PREC_F64) return BR_EINVAL;
  return BR_OK;
}

// Launch shape, shared-memory attribute, queue reset and launch of both LM entry points
// (arguments already checked by lm_check); `queue` is BR_LM_SCRATCH_BYTES of device memory.
static int lm_launch(const br_ik_batch_t& b, const br_ik_settings_t& settings, const br_ik_result_t& result,
                     int32_t warps_per_cta, void* queue, cudaStream_t s) {
  LmParams p = {};
  p.s = settings;
  p.b = b;
  p.r = result;
  const bool f64 = settings.precision == BR_PREC_F64;
  int warp_floats = 0;
  for (int c = 0; c < b.n_classes; ++c) {
    const int st = validate_tree(&b.trees[c]);
    if (st) return st;
    if (!b.trees[c].dof_sched) return BR_EINVAL;           // the factorization's level schedule
    const int T = b.team_size[c];
    if (T != kLmTeam) return BR_EINVAL;                    // the kernel is built for 32-lane teams
    p.trees[c] = b.trees[c];
    p.team[c] = T;
    const br_tree_t& tc = b.trees[c];
    const int f = (32 / T) * TeamLayout(tc.njoints, tc.nq, tc.nv, b.max_targets, T, tc.dof_entries, tc.dof_depth,
                                        tc.rounds, f64 ? 2 : 1).total;
    if (f > warp_floats) warp_floats = f;
  }
  p.warp_floats = warp_floats;
  p.queue = reinterpret_cast<int32_t*>(queue);
  const DeviceInfo& dev = device_info();
  if (dev.device < 0 || dev.device >= 64) return BR_EINVAL;
  int wpc = warps_per_cta;
  size_t bytes = (size_t)wpc * warp_floats * sizeof(float);
  while ((int64_t)bytes > dev.max_smem_optin && wpc > 1) {
    wpc >>= 1;
    bytes = (size_t)wpc * warp_floats * sizeof(float);
  }
  if ((int64_t)bytes > dev.max_smem_optin) return BR_ETOOBIG;
  bool general = b.target_kind != nullptr || settings.kernel != BR_KERNEL_L2;
  for (int c = 0; c < b.n_classes; ++c) general |= (b.trees[c].kinds & ~kBasicKinds) != 0 || b.trees[c].kinds == 0;
  auto kern = f64 ? (general ? lm_solve_kernel<true, true> : lm_solve_kernel<false, true>)
                 : (general ? lm_solve_kernel<true, false> : lm_solve_kernel<false, false>);
  {
    std::lock_guard<std::mutex> lock(g_lm_mu);
    int& have = g_smem_allowed[(f64 ? 2 : 0) + (general ? 1 : 0)][dev.device];
    if ((int)bytes > have) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      if (e != cudaSuccess) return (int)e;
      have = (int)bytes;
    }
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpc * kWarp, bytes);
  if (per_sm < 1) per_sm = 1;
  const int64_t need = (b.n_items + wpc - 1) / wpc;
  const int64_t cap = (int64_t)per_sm * dev.sms;
  const int grid = (int)(need < cap ? need : cap);
  cudaError_t e = cudaMemsetAsync(queue, 0, BR_LM_SCRATCH_BYTES, s);  // the queue counter starts at zero
  if (e != cudaSuccess) return (int)e;
  kern<<<grid, wpc * kWarp, bytes, s>>>(p);
  return (int)cudaGetLastError();
}

extern "C" int br_lm_solve(const br_ik_batch_t* batch, const br_ik_settings_t* settings, br_ik_result_t* result,
                           int32_t warps_per_cta, void* scratch, int64_t scratch_bytes, void* stream) {
  if (batch && (!scratch || scratch_bytes < BR_LM_SCRATCH_BYTES)) return BR_EINVAL;
  const int st = lm_check(batch, settings, result, warps_per_cta);
  if (st) return st == kLmNothing ? BR_OK : st;
  return lm_launch(*batch, *settings, *result, warps_per_cta, scratch, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of br_lm_solve.
//
// br_lm_solve needs 16 bytes of device scratch (its work-queue counter) from the
// caller.  Some callers cannot provide it because they cannot call cudaMalloc at
// all: an IK call made from a robot controller's real-time loop, where a device
// allocation can block for milliseconds and serialise the whole device; or a host
// program that receives its input and output buffers from a framework and has no
// CUDA allocator of its own.  br_lm_solve_noalloc runs the same kernel with the
// scratch taken from the file-scope array below, so a call allocates nothing.
//
// The array exists once per device that loads this library and lives until the
// process exits.  All calls on a device share it: two calls that run at the same
// time on the GPU (e.g. on two streams) race on the work queue and must not
// overlap.  Each call zeroes the part it uses before its launch.  The array's device
// address is looked up on the first call on each device and kept: a cudaDeviceReset
// between calls reloads the module at another address and is not supported.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_lm_noalloc_scratch[BR_LM_NOALLOC_SCRATCH_BYTES];

namespace {
void* g_noalloc_ptr[64] = {};  // device address of g_lm_noalloc_scratch, per device ordinal
}  // namespace

// Host code cannot use g_lm_noalloc_scratch as a device address; look the address
// up once per device, with that device current (the first call on each device).
static int noalloc_scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= 64) return BR_EINVAL;
  std::lock_guard<std::mutex> lock(g_lm_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lm_noalloc_scratch);
    if (e != cudaSuccess) return (int)e;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return BR_OK;
}

extern "C" int br_lm_solve_noalloc(const br_ik_batch_t* batch, const br_ik_settings_t* settings,
                                   br_ik_result_t* result, int32_t warps_per_cta, void* stream) {
  static_assert(BR_LM_SCRATCH_BYTES <= BR_LM_NOALLOC_SCRATCH_BYTES, "the static scratch is too small");
  const int st = lm_check(batch, settings, result, warps_per_cta);
  if (st) return st == kLmNothing ? BR_OK : st;
  void* scratch = nullptr;
  const int sa = noalloc_scratch_address(&scratch);
  if (sa) return sa;
  return lm_launch(*batch, *settings, *result, warps_per_cta, scratch, (cudaStream_t)stream);
}

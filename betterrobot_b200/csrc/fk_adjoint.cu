// fk_adjoint.cu — pose loss through forward kinematics and its hand-written adjoint.
//
// Loss per configuration:  L(q) = sum_f w_f |log(T_f^-1 * oMf(q))|^2
// (the reference obtains dL/dq by torch autograd through every SE3 op of
// src/better_robot/kinematics/forward.py:73-135 and lie/_torch_native_backend.py).
//
// Adjoint, one warp per configuration (two configurations per pass of the warp where their
// frames fit one lane each: the per-frame stage then runs on both at once):
//   * g_f = 2 w_f Jr^-1(xi_f)^T xi_f is dL/d(body twist of frame f), with the exact
//     SE3 Jr^-1 (closed form jr_inv_T_xi; autograd differentiates se3_log exactly);
//   * F_f = Ad(oMf^-1)^T g_f = [R g_lin; p x (R g_lin) + R g_ang] is the same
//     sensitivity as a wrench at the world origin;
//   * dL/dv_c = sum_{f : c supports f} <S_c, F_f> = <S_c, W_j> with S_c the world twist
//     of tangent column c ([o x a; a] rotation, [a; 0] translation) and W_j the summed
//     wrench of the frames that c's joint j moves — a reverse accumulation over the tree
//     without any per-joint tape;
//   * revolute / prismatic / translation: dL/dq = dL/dv; free-flyer and spherical: the
//     body twist of the joint maps to raw q = [t, quat] through R (translation) and the
//     normalisation of the quaternion ((I - u u^T)/|quat| and du -> 2 vec(u* (x) du));
//     unbounded revolute: th = atan2(s, c); planar: [x, y] through R, the angle through
//     the reference's half-angle formula (dth/dc = -1/sin th, no dependence on s).
// World joint placements are either recomputed from q (no saved state) or read
// from the forward pass (store mode, [B, njoints, 7]).
#include <cuda_runtime.h>
#include <stdint.h>

#include "br_common.cuh"
#include "br_fk.cuh"
#include "br_lie.cuh"

namespace br {

struct LossParams {
  const float* q;          // [B, nq]
  const float* targets;    // [B, nf, 7]
  const float* weights;    // [nf] or [B, nf]
  const float* grad_loss;  // [B] (backward)
  const float* oMi_in;     // [B, nj, 7] (backward, store mode) or null
  float* loss;             // [B] (forward)
  float* oMi_out;          // [B, nj, 7] (forward, store mode) or null
  float* grad_q;           // [B, nq] (backward)
  int64_t batch;
  int32_t nf;
  int32_t weights_per_config;
  int32_t frames[BR_MAX_TARGETS];
};

struct LossLayout {
  int parent, jtype, idxq, axis, place, cjoint, ckind, caxis, fparent, fplace, fsup;
  int cta_floats;
  int in0, in1, poseT, poseQ, anc, F, W, gv, stage;
  int pair;   // configurations per pass (2 or 1)
  int inlen;  // floats of one configuration's inputs (16-byte multiple)
  int warp_floats;
  // A warp's slice with two configurations per pass above this many floats would leave one
  // 8-warp CTA per SM instead of two (the humanoid at 12 frames takes 2,644).
  static constexpr int kPairMaxWarpFloats = 3456;
  __host__ __device__ LossLayout(int nj, int nq, int nv, int nf) {
    int o = 0;
    auto take = [&](int n) { int r = o; o += round4(n); return r; };
    parent = take(nj); jtype = take(nj); idxq = take(nj); axis = take(4 * nj); place = take(8 * nj);
    cjoint = take(nv); ckind = take(nv); caxis = take(4 * nv);
    fparent = take(nf); fplace = take(8 * nf); fsup = take(2 * nf);
    cta_floats = o;
    inlen = round4(nq + 7 * nj + 7 * nf);
    // two configurations per pass when both configurations' frames fit one lane each and the
    // slice stays small enough, else one
    for (pair = 2 * nf <= 32 ? 2 : 1;; pair = 1) {
      o = 0;
      // the inputs of a pass's configurations (q, stored oMi, targets), double buffered: the
      // next pass's are copied in (cp.async) while this one is computed
      in0 = take(pair * inlen); in1 = take(pair * inlen);
      poseT = take(pair * 4 * nj); poseQ = take(pair * 4 * nj); anc = take(nj);
      F = take(pair * 8 * nf);  // world wrench per frame (f.xyz, pad, tau.xyz, pad), per configuration
      W = take(8 * nj);         // summed wrench of the frames each joint moves (same layout)
      gv = take(nv);            // dL/dv
      stage = take(nj * 7);     // oMi staging (store mode)
      warp_floats = o;
      if (pair == 1 || warp_floats <= kPairMaxWarpFloats) break;
    }
  }
};

template <bool kBackward>
__global__ void __launch_bounds__(256, 2) pose_loss_kernel(const br_tree_t tree, const LossParams p) {
  extern __shared__ __align__(16) float smem[];
  const int nj = tree.njoints, nq = tree.nq, nv = tree.nv, nf = p.nf;
  const LossLayout L(nj, nq, nv, nf);
  int* s_parent = reinterpret_cast<int*>(smem + L.parent);
  int* s_jtype = reinterpret_cast<int*>(smem + L.jtype);
  int* s_idxq = reinterpret_cast<int*>(smem + L.idxq);
  float* s_axis = smem + L.axis;
  float* s_place = smem + L.place;
  int* s_cjoint = reinterpret_cast<int*>(smem + L.cjoint);
  int* s_ckind = reinterpret_cast<int*>(smem + L.ckind);
  float* s_caxis = smem + L.caxis;
  int* s_fparent = reinterpret_cast<int*>(smem + L.fparent);
  float* s_fplace = smem + L.fplace;
  unsigned long long* s_fsup = reinterpret_cast<unsigned long long*>(smem + L.fsup);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  for (int i = threadIdx.x; i < nj; i += blockDim.x) {
    s_parent[i] = tree.parent[i];
    s_jtype[i] = tree.jtype[i];
    s_idxq[i] = tree.idx_q[i];
    for (int k = 0; k < 4; ++k) s_axis[4 * i + k] = tree.axis[4 * i + k];
    for (int k = 0; k < 8; ++k) s_place[8 * i + k] = tree.placement[8 * i + k];
  }
  for (int c = threadIdx.x; c < nv; c += blockDim.x) {
    s_cjoint[c] = tree.col_joint[c];
    s_ckind[c] = tree.col_kind[c];
    for (int k = 0; k < 4; ++k) s_caxis[4 * c + k] = tree.col_axis[4 * c + k];
  }
  for (int f = threadIdx.x; f < nf; f += blockDim.x) {
    const int id = p.frames[f];
    s_fparent[f] = tree.frame_parent[id];
    for (int k = 0; k < 8; ++k) s_fplace[8 * f + k] = tree.frame_placement[8 * id + k];
  }
  __syncthreads();
  // joints that move each frame: bit j set iff joint j supports the frame's parent joint
  for (int f = threadIdx.x; f < nf; f += blockDim.x) s_fsup[f] = tree.support[s_fparent[f]];
  __syncthreads();

  float* w = smem + L.cta_floats + warp * L.warp_floats;
  int* wanc = reinterpret_cast<int*>(w + L.anc);
  float* wW = w + L.W;
  float* wg = w + L.gv;
  float* wst = w + L.stage;
  const int64_t stride = (int64_t)gridDim.x * wpc;
  const bool stored = kBackward && p.oMi_in;
  const int o_pose = nq, o_tgt = nq + (stored ? 7 * nj : 0);   // offsets in an input buffer
  // Configurations b and b + stride are taken as a pair when both fit the frame stage's lanes
  // (2 nf <= 32): their FK, per-joint and per-column stages run one after the other over the
  // whole warp, the per-frame stage (one lane per frame) over both at once.  Pose set, wrench
  // set and input buffer hp belong to configuration b + hp * stride.
  const int pair = L.pair;
  const int64_t step = stride * pair;
  // queue the copies of configuration bb's inputs into `dst` (nothing past the end of the
  // batch): 4-byte cp.async, the rows are 4-byte aligned only
  auto prefetch = [&](int64_t bb, float* dst) {
    if (bb < p.batch) {
      const float* qb = p.q + bb * nq;
      for (int i = lane; i < nq; i += kWarp) cp_async4(dst + i, qb + i);
      if (stored) {
        const float* ob = p.oMi_in + bb * (int64_t)nj * 7;
        for (int i = lane; i < nj * 7; i += kWarp) cp_async4(dst + o_pose + i, ob + i);
      }
      const float* tb = p.targets + bb * (int64_t)nf * 7;
      for (int i = lane; i < nf * 7; i += kWarp) cp_async4(dst + o_tgt + i, tb + i);
    }
  };
  float* cur = w + L.in0;                  // this pass's inputs; the other buffers: the next pass's
  float* nxt = w + L.in1;
  int64_t b = (int64_t)blockIdx.x * wpc + warp;
  for (int hp = 0; hp < pair; ++hp) prefetch(b + hp * stride, cur + hp * L.inlen);
  cp_async_commit();                       // one commit group per pass
  for (; b < p.batch; b += step) {
    __syncwarp();                          // every lane is done with the buffers refilled next
    for (int hp = 0; hp < pair; ++hp) prefetch(b + step + hp * stride, nxt + hp * L.inlen);
    cp_async_commit();
    cp_async_wait_groups<1>();             // this pass's copies (all but the newest group)
    __syncwarp();
    const float* wq0 = cur;
    { float* t = cur; cur = nxt; nxt = t; }
    const int np = (pair == 2 && b + stride < p.batch) ? 2 : 1;
    for (int hp = 0; hp < np; ++hp) {
      const int64_t bh = b + hp * stride;
      const float* wqh = wq0 + hp * L.inlen;
      float* wpT = w + L.poseT + hp * 4 * nj;
      float* wpQ = w + L.poseQ + hp * 4 * nj;
      if (stored) {
        const float* ob = wqh + o_pose;
        for (int i = lane; i < nj * 7; i += kWarp) {
          const int j = i / 7, c = i - 7 * j;
          if (c < 3) wpT[4 * j + c] = ob[i];
          else wpQ[4 * j + c - 3] = ob[i];
        }
        __syncwarp();
      } else {
        // forward kinematics by pointer jumping (see fk_jac.cu)
        for (int j = lane; j < nj; j += kWarp) {
          store_split(wpT, wpQ, j, local_transform(s_jtype[j], load_pose8(s_place + 8 * j), s_axis + 4 * j,
                                                   wqh + s_idxq[j]));
          wanc[j] = s_parent[j];
        }
        __syncwarp();
        for (int r = 0; r < tree.rounds; ++r) {
          Pose A[2], Tj[2];
          int aa[2], an[2];
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const int j = lane + kWarp * k;
            an[k] = (j < nj) ? wanc[j] : -1;
            if (an[k] >= 0) {
              A[k] = load_split(wpT, wpQ, an[k]);
              Tj[k] = load_split(wpT, wpQ, j);
              aa[k] = wanc[an[k]];
            }
          }
          __syncwarp();
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const int j = lane + kWarp * k;
            if (an[k] >= 0) {
              store_split(wpT, wpQ, j, compose(A[k], Tj[k]));
              wanc[j] = aa[k];
            }
          }
          __syncwarp();
        }
        if (!kBackward && p.oMi_out) {
          for (int j = lane; j < nj; j += kWarp) store_pose7(wst + 7 * j, load_split(wpT, wpQ, j));
          __syncwarp();
          warp_copy(p.oMi_out + bh * (int64_t)nj * 7, wst, nj * 7, lane);
          __syncwarp();
        }
      }
    }
    // per-frame residual, loss and (backward) world wrench; frame f of the pair's second
    // configuration on lane nf + f
    float acc0 = 0.f, acc1 = 0.f;
    for (int i = lane; i < np * nf; i += kWarp) {
      const int hp = i >= nf ? 1 : 0;
      const int f = i - hp * nf;
      const int64_t bh = b + hp * stride;
      const Pose Tf = compose(load_split(w + L.poseT + hp * 4 * nj, w + L.poseQ + hp * 4 * nj, s_fparent[f]),
                              load_pose8(s_fplace + 8 * f));
      const float* tp = wq0 + hp * L.inlen + o_tgt + 7 * f;
      const Pose Tt{f3(tp[0], tp[1], tp[2]), make_float4(tp[3], tp[4], tp[5], tp[6])};
      float3 v, om;
      se3_log(compose(inverse(Tt), Tf), v, om);
      const float wf = __ldg(p.weights + (p.weights_per_config ? bh * nf + f : f));
      const float lf = wf * (dot(v, v) + dot(om, om));
      if (hp) acc1 += lf; else acc0 += lf;
      if (kBackward) {
        float3 gl, ga;
        jr_inv_T_xi(v, om, gl, ga);
        const float s2 = 2.f * wf;
        const float3 fw = qrot(Tf.q, scale(gl, s2));
        const float3 tau = add(cross(Tf.t, fw), qrot(Tf.q, scale(ga, s2)));
        float* wF = w + L.F + hp * 8 * nf;
        *reinterpret_cast<float4*>(wF + 8 * f) = make_float4(fw.x, fw.y, fw.z, 0.f);
        *reinterpret_cast<float4*>(wF + 8 * f + 4) = make_float4(tau.x, tau.y, tau.z, 0.f);
      }
    }
    if (!kBackward) {
      // the second configuration's terms moved to lanes 0..nf-1 first, so that both sums
      // take the same order (that of a configuration processed alone)
      if (pair == 2) {
        const float m1 = __shfl_sync(0xffffffffu, acc1, (lane + nf) & (kWarp - 1));
        acc1 = lane + nf < kWarp ? m1 : 0.f;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        acc0 += __shfl_xor_sync(0xffffffffu, acc0, o);
        acc1 += __shfl_xor_sync(0xffffffffu, acc1, o);
      }
      if (lane == 0) {
        p.loss[b] = acc0;
        if (np == 2) p.loss[b + stride] = acc1;
      }
      continue;
    }
    __syncwarp();
    for (int hp = 0; hp < np; ++hp) {
      const int64_t bh = b + hp * stride;
      const float* wqh = wq0 + hp * L.inlen;
      const float* wF = w + L.F + hp * 8 * nf;
      const float* wpT = w + L.poseT + hp * 4 * nj;
      const float* wpQ = w + L.poseQ + hp * 4 * nj;
      // dL/dv_c = sum over the frames f that column c moves of <S_c, F_f> = <S_c, W_j>, where
      // W_j sums F_f over the frames that c's joint j moves: one sum per joint, one dot per column
      for (int j = lane; j < nj; j += kWarp) {
        float4 sf = make_float4(0.f, 0.f, 0.f, 0.f), st = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int f = 0; f < nf; ++f) {
          if ((s_fsup[f] >> j) & 1ull) {
            const float4 fw = *reinterpret_cast<const float4*>(wF + 8 * f);
            const float4 tq = *reinterpret_cast<const float4*>(wF + 8 * f + 4);
            sf.x += fw.x; sf.y += fw.y; sf.z += fw.z;
            st.x += tq.x; st.y += tq.y; st.z += tq.z;
          }
        }
        *reinterpret_cast<float4*>(wW + 8 * j) = sf;
        *reinterpret_cast<float4*>(wW + 8 * j + 4) = st;
      }
      __syncwarp();
      const float go = __ldg(p.grad_loss + bh);
      for (int c = lane; c < nv; c += kWarp) {
        const int j = s_cjoint[c];
        const Pose Tj = load_split(wpT, wpQ, j);
        const float3 a = qrot(Tj.q, f3(s_caxis[4 * c], s_caxis[4 * c + 1], s_caxis[4 * c + 2]));
        const float3 m = s_ckind[c] == 0 ? cross(Tj.t, a) : a;  // linear part of the world twist
        const float3 an = s_ckind[c] == 0 ? a : f3(0.f, 0.f, 0.f);
        const float4 fw = *reinterpret_cast<const float4*>(wW + 8 * j);
        const float4 tq = *reinterpret_cast<const float4*>(wW + 8 * j + 4);
        wg[c] = (dot(m, f3(fw.x, fw.y, fw.z)) + dot(an, f3(tq.x, tq.y, tq.z))) * go;
      }
      __syncwarp();
      float* gq = p.grad_q + bh * nq;
      for (int j = lane; j < nj; j += kWarp) {
        const int jt = s_jtype[j];
        const int iq = s_idxq[j];
        if (jt == BR_JOINT_REVOLUTE || jt == BR_JOINT_PRISMATIC) {
          gq[iq] = wg[tree.idx_v[j]];
        } else if (jt == BR_JOINT_TRANSLATION) {                     // q is the body translation
          const int iv = tree.idx_v[j];
          gq[iq] = wg[iv]; gq[iq + 1] = wg[iv + 1]; gq[iq + 2] = wg[iv + 2];
        } else if (jt == BR_JOINT_REVOLUTE_UNBOUNDED) {
          // th = atan2(s, c) (revolute.py:206-211): dth/dc = -s / r^2, dth/ds = c / r^2
          const float g = wg[tree.idx_v[j]];
          const float c = wqh[iq], sn = wqh[iq + 1];
          const float r2 = fmaxf(c * c + sn * sn, 1e-30f);
          gq[iq] = -g * sn / r2;
          gq[iq + 1] = g * c / r2;
        } else if (jt == BR_JOINT_PLANAR) {
          // T = ([x, y, 0], Rz(th)) with cos(th/2) = sqrt((1+c)/2), sin(th/2) = sqrt((1-c)/2) sign(s)
          // (planar.py:20-41): body twist = (R^T [dx, dy, 0], e_z dth), dth/dc = -1 / sin(th),
          // and th does not depend on s away from s = 0
          const int iv = tree.idx_v[j];
          const float c = wqh[iq + 2], sn = wqh[iq + 3];
          const float4 hq = planar_quat(c, sn);
          const float ct = hq.w * hq.w - hq.z * hq.z, st = 2.f * hq.z * hq.w;
          const float g0 = wg[iv], g1 = wg[iv + 1], g2 = wg[iv + 2];
          gq[iq] = ct * g0 - st * g1;
          gq[iq + 1] = st * g0 + ct * g1;
          gq[iq + 2] = -g2 / st;
          gq[iq + 3] = 0.f;
        } else if (jt == BR_JOINT_FREE_FLYER || jt == BR_JOINT_SPHERICAL) {
          // free-flyer [t, quat] / spherical [quat]: the quaternion's body rotation
          const bool ff = jt == BR_JOINT_FREE_FLYER;
          const int iv = tree.idx_v[j];
          const int qo = ff ? iq + 3 : iq;                          // first quaternion slot
          const int vo = ff ? iv + 3 : iv;                          // first rotation column
          const float4 qr = make_float4(wqh[qo], wqh[qo + 1], wqh[qo + 2], wqh[qo + 3]);
          const float4 u = qnormalize(qr);
          const float n = fmaxf(sqrtf(qr.x * qr.x + qr.y * qr.y + qr.z * qr.z + qr.w * qr.w), 1e-8f);
          const float3 ga = f3(wg[vo], wg[vo + 1], wg[vo + 2]);
          // quaternion: delta_ang = 2 vec(u* (x) du), du = (I - u u^T) dquat / n
          float4 h;
          h.x = u.w * ga.x - u.z * ga.y + u.y * ga.z;
          h.y = u.z * ga.x + u.w * ga.y - u.x * ga.z;
          h.z = -u.y * ga.x + u.x * ga.y + u.w * ga.z;
          h.w = -u.x * ga.x - u.y * ga.y - u.z * ga.z;
          const float uh = u.x * h.x + u.y * h.y + u.z * h.z + u.w * h.w;
          const float s = 2.f / n;
          if (ff) {
            const float3 gt = qrot(u, f3(wg[iv], wg[iv + 1], wg[iv + 2]));  // translation: delta_lin = R^T dt
            gq[iq] = gt.x; gq[iq + 1] = gt.y; gq[iq + 2] = gt.z;
          }
          gq[qo] = s * (h.x - u.x * uh);
          gq[qo + 1] = s * (h.y - u.y * uh);
          gq[qo + 2] = s * (h.z - u.z * uh);
          gq[qo + 3] = s * (h.w - u.w * uh);
        }
      }
      __syncwarp();
    }
  }
  cp_async_wait_groups<0>();               // the (empty) last group
}

template <bool kBackward>
static int launch_loss(const br_tree_t& tree, const LossParams& p, int wpc, cudaStream_t stream) {
  if (p.batch == 0) return BR_OK;
  const LossLayout L(tree.njoints, tree.nq, tree.nv, p.nf);
  const DeviceInfo& dev = device_info();
  size_t bytes = (size_t)(L.cta_floats + wpc * L.warp_floats) * sizeof(float);
  while ((int)bytes > dev.max_smem_optin && wpc > 1) {
    wpc >>= 1;
    bytes = (size_t)(L.cta_floats + wpc * L.warp_floats) * sizeof(float);
  }
  auto kern = pose_loss_kernel<kBackward>;
  static int configured[16] = {0};
  if ((int)bytes > configured[dev.device & 15]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    configured[dev.device & 15] = (int)bytes;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpc * kWarp, bytes);
  if (per_sm < 1) per_sm = 1;
  const int64_t need = (p.batch + wpc - 1) / wpc;
  const int64_t cap = (int64_t)per_sm * dev.sms;
  kern<<<(int)(need < cap ? need : cap), wpc * kWarp, bytes, stream>>>(tree, p);
  return (int)cudaGetLastError();
}

static int fill_loss(const br_tree_t* tree, LossParams& p, const int32_t* frame_ids, int32_t n_frames) {
  int st = validate_tree(tree);
  if (st) return st;
  if (n_frames < 1 || !frame_ids) return BR_EINVAL;
  if (n_frames > BR_MAX_TARGETS) return BR_ETOOBIG;
  for (int i = 0; i < n_frames; ++i) {
    if (frame_ids[i] < 0 || frame_ids[i] >= tree->nframes) return BR_EINVAL;
    p.frames[i] = frame_ids[i];
  }
  p.nf = n_frames;
  return BR_OK;
}

}  // namespace br

using namespace br;

// Joint kinds whose raw-q chain rule the backward implements: every kind of the tree table.
static bool adjoint_kinds_ok(const br_tree_t* t) {
  const int ok = (1 << (BR_JOINT_TRANSLATION + 1)) - 1;
  return t && t->kinds != 0 && (t->kinds & ~ok) == 0;
}

extern "C" int br_pose_loss(const br_tree_t* tree, const float* q, int64_t batch, const int32_t* frame_ids,
                            int32_t n_frames, const float* targets, const float* weights,
                            int32_t weights_per_config, float* loss, float* joint_pose_world, void* stream) {
  LossParams p = {};
  int st = fill_loss(tree, p, frame_ids, n_frames);
  if (st) return st;
  if (!adjoint_kinds_ok(tree)) return BR_EINVAL;
  if (batch < 0 || (batch > 0 && (!q || !targets || !weights || !loss))) return BR_EINVAL;
  p.q = q; p.targets = targets; p.weights = weights; p.loss = loss; p.oMi_out = joint_pose_world;
  p.batch = batch; p.weights_per_config = weights_per_config != 0;
  return launch_loss<false>(*tree, p, 8, (cudaStream_t)stream);
}

extern "C" int br_pose_loss_backward(const br_tree_t* tree, const float* q, const float* joint_pose_world,
                                     int64_t batch, const int32_t* frame_ids, int32_t n_frames,
                                     const float* targets, const float* weights, int32_t weights_per_config,
                                     const float* grad_loss, float* grad_q, void* stream) {
  LossParams p = {};
  int st = fill_loss(tree, p, frame_ids, n_frames);
  if (st) return st;
  if (!adjoint_kinds_ok(tree)) return BR_EINVAL;
  if (batch < 0 || (batch > 0 && (!q || !targets || !weights || !grad_loss || !grad_q))) return BR_EINVAL;
  p.q = q; p.oMi_in = joint_pose_world; p.targets = targets; p.weights = weights;
  p.grad_loss = grad_loss; p.grad_q = grad_q; p.batch = batch; p.weights_per_config = weights_per_config != 0;
  return launch_loss<true>(*tree, p, 8, (cudaStream_t)stream);
}

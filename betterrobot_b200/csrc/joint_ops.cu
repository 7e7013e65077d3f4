// joint_ops.cu — batched configuration-space retraction and difference.
//
// integrate:  q' = q (+) v   (Model.integrate, src/better_robot/data_model/model.py:160-174):
//   revolute / prismatic / translation  q' = q + v       (revolute.py:46-48, translation.py:40-41)
//   free-flyer            q' = normalize(q * exp(v))     (free_flyer.py:47-51)
//   spherical             q' = normalize(q * exp(v))     (spherical.py:52-56)
//   planar, unbounded     theta' = atan2(sin, cos) + v   (planar.py:61-68, revolute.py:223-231)
// difference: v = q1 (-) q0  (Model.difference, model.py:176-190):
//   revolute / prismatic / translation  v = q1 - q0      (revolute.py:51-53)
//   free-flyer            v = log(q0^-1 * q1)            (free_flyer.py:53-57)
//   spherical             v = log(normalize(q0^-1 q1))   (spherical.py:58-62)
//   planar, unbounded     atan2(q1) - atan2(q0)          (planar.py:70-76, revolute.py:233-237)
//
// Layout: a warp owns a tile of 32 consecutive configurations.  Their rows of every
// input are one contiguous slab, copied into the warp's shared memory with 16-byte
// cp.async copies (all of a tile's copies in flight at once); the slots of the other kinds
// (free-flyer, spherical, planar, unbounded) are then computed one configuration per lane (the float64 exp / log runs on 32 lanes at once),
// and the output slab is written with float4 stores, each lane producing 4 consecutive
// outputs.  Memory bound: 4 * (nq + nv + nq) bytes per configuration for integrate,
// 4 * (nq + nq + nv) for difference.  Pointers that are not 16-byte aligned take the
// same path with 4-byte loads and stores (kVec = false).
#include <cuda_runtime.h>
#include <stdint.h>

#include "br_common.cuh"
#include "br_fk.cuh"
#include "br_lie.cuh"

namespace br {

struct JointOpParams {
  const float* a;   // q (integrate) or q0 (difference)        [B, nq]
  const float* b;   // v (integrate, [B, nv]) or q1 (difference, [B, nq])
  float* out;       // q' [B, nq] or v [B, nv]
  int64_t batch;
  int32_t n_active; // joints with nq > 0
  int32_t diff;     // 0 integrate, 1 difference
};

constexpr int kJointOpsWarps = 4;

// Floats of shared memory one warp stages.  integrate: two input tiles (the next one is
// copied while this one is computed).  difference: one input tile, whose q0 rows also take
// the outputs of the joints computed per lane (a joint's nv outputs overwrite the first nv
// of its own nq >= nv slots); a second tile would halve its warps per SM (its float64 logs
// make it compute heavy: measured at 1 M humanoid configurations, 104 -> 162 us).
__host__ __device__ inline int joint_ops_in_floats(int nq, int nv, bool diff) { return 32 * (diff ? 2 * nq : nq + nv); }
__host__ __device__ inline int joint_ops_warp_floats(int nq, int nv, bool diff) {
  return diff ? joint_ops_in_floats(nq, nv, diff) : 2 * joint_ops_in_floats(nq, nv, diff);
}

__device__ __forceinline__ DPose dpose7(const float* p) {
  return DPose{d3(p[0], p[1], p[2]), make_double4(p[3], p[4], p[5], p[6])};
}

template <bool kVec>
__device__ __forceinline__ void slab_in(float* s, const float* __restrict__ g, int n, int lane) {
  int done = 0;
  if (kVec) {
    const int n4 = n >> 2;
    for (int i = lane; i < n4; i += 32) cp_async16(s + 4 * i, g + 4 * i);
    done = n4 << 2;
  }
  for (int i = done + lane; i < n; i += 32) s[i] = g[i];
}

template <bool kVec>
__global__ void __launch_bounds__(32 * kJointOpsWarps) joint_ops_kernel(const br_tree_t tree,
                                                                        const int32_t* __restrict__ active,
                                                                        const JointOpParams p) {
  extern __shared__ __align__(16) float slabs[];
  __shared__ int16_t vmap[BR_MAX_NQ];     // q slot -> v slot of a 1:1 joint, -1 for other slots
  __shared__ int16_t qmap[BR_MAX_NV];     // v slot -> q slot k of a 1:1 joint (k), or of the q0 slot that
                                          // holds a per-lane joint's output (-k - 1)
  __shared__ int16_t ffq[BR_MAX_JOINTS];  // q / v offsets and kind of the joints handled per lane
  __shared__ int16_t ffv[BR_MAX_JOINTS];   // (free-flyer, spherical, planar, unbounded revolute)
  __shared__ int8_t ffk[BR_MAX_JOINTS];
  __shared__ int nff;
  const int nq = tree.nq, nv = tree.nv;
  for (int k = threadIdx.x; k < nq; k += blockDim.x) vmap[k] = -1;
  for (int k = threadIdx.x; k < nv; k += blockDim.x) qmap[k] = -1;
  if (threadIdx.x == 0) nff = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < p.n_active; i += blockDim.x) {
    const int j = active[i];
    const int iq = tree.idx_q[j], iv = tree.idx_v[j];
    const int jt = tree.jtype[j];
    if (joint_is_vector(jt)) {
      for (int k = 0; k < joint_nv(jt); ++k) {
        vmap[iq + k] = (int16_t)(iv + k);
        qmap[iv + k] = (int16_t)(iq + k);
      }
    } else {
      for (int k = 0; k < joint_nv(jt); ++k) qmap[iv + k] = (int16_t)(-(iq + k) - 1);
      const int s = atomicAdd(&nff, 1);
      ffq[s] = (int16_t)iq;
      ffv[s] = (int16_t)iv;
      ffk[s] = (int8_t)jt;
    }
  }
  __syncthreads();
  const bool diff = p.diff != 0;
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const int lb = diff ? nq : nv;  // floats per configuration of b
  const int lo = diff ? nv : nq;  // floats per configuration of out
  const int IN = joint_ops_in_floats(nq, nv, diff);
  float* base = slabs + (size_t)(threadIdx.x >> 5) * joint_ops_warp_floats(nq, nv, diff);
  const bool dbl = kVec && !diff; // integrate with 16-byte copies: next tile in flight
  const int64_t tiles = (p.batch + 31) >> 5;
  const int64_t step = (int64_t)gridDim.x * warps;
  const int n_ff = nff;
  auto fetch = [&](int64_t t, float* buf) {  // the tile's rows of both inputs into buf
    const int64_t b = t << 5;
    const int c = p.batch - b < 32 ? (int)(p.batch - b) : 32;
    slab_in<kVec>(buf, p.a + b * nq, c * nq, lane);
    slab_in<kVec>(buf + 32 * nq, p.b + b * lb, c * lb, lane);
  };
  int64_t tile = (int64_t)blockIdx.x * warps + (threadIdx.x >> 5);
  if (dbl && tile < tiles) fetch(tile, base);
  if (dbl) cp_async_commit();
  for (int k = 0; tile < tiles; tile += step, ++k) {
    const int64_t b0 = tile << 5;
    const int cnt = p.batch - b0 < 32 ? (int)(p.batch - b0) : 32;
    float* A = dbl ? base + (k & 1) * IN : base;
    float* Bs = A + 32 * nq;
    if (dbl) {  // the next tile's copies are issued before this one is computed
      if (tile + step < tiles) fetch(tile + step, base + ((k + 1) & 1) * IN);
      cp_async_commit();
      cp_async_wait_groups<1>();
    } else {
      fetch(tile, A);
      if (kVec) cp_async_wait_all();
    }
    __syncwarp();
    if (lane < cnt) {
      for (int f = 0; f < n_ff; ++f) {
        const int iq = ffq[f], iv = ffv[f], jt = ffk[f];
        float* qa = A + lane * nq + iq;
        if (!diff) {
          const float* v = Bs + lane * nv + iv;
          if (jt == BR_JOINT_FREE_FLYER) {
            DPose n = dcompose(dpose7(qa), dse3_exp(d3(v[0], v[1], v[2]), d3(v[3], v[4], v[5])));
            n.q = dqnormalize(n.q);
            qa[0] = (float)n.t.x; qa[1] = (float)n.t.y; qa[2] = (float)n.t.z;
            qa[3] = (float)n.q.x; qa[4] = (float)n.q.y; qa[5] = (float)n.q.z; qa[6] = (float)n.q.w;
          } else if (jt == BR_JOINT_SPHERICAL) {  // normalize(q * exp(v)), spherical.py:52-56
            const double4 n = dqnormalize(dqmul(make_double4(qa[0], qa[1], qa[2], qa[3]),
                                                dse3_exp(d3(0.0, 0.0, 0.0), d3(v[0], v[1], v[2])).q));
            qa[0] = (float)n.x; qa[1] = (float)n.y; qa[2] = (float)n.z; qa[3] = (float)n.w;
          } else {                                // planar.py:61-68, revolute.py:223-231
            const int k = jt == BR_JOINT_PLANAR ? 2 : 0;
            double s, c;
            sincos(atan2((double)qa[k + 1], (double)qa[k]) + (double)v[k], &s, &c);
            if (jt == BR_JOINT_PLANAR) {
              qa[0] = qa[0] + v[0];
              qa[1] = qa[1] + v[1];
            }
            qa[k] = (float)c;
            qa[k + 1] = (float)s;
          }
        } else {
          // outputs in place of the joint's own q0 slots (each read before it is written)
          const float* qb = Bs + lane * nq + iq;
          float* o = qa;
          if (jt == BR_JOINT_FREE_FLYER) {
            double3 v, w;
            dse3_log(dcompose(dinverse(dpose7(qa)), dpose7(qb)), v, w);
            o[0] = (float)v.x; o[1] = (float)v.y; o[2] = (float)v.z;
            o[3] = (float)w.x; o[4] = (float)w.y; o[5] = (float)w.z;
          } else if (jt == BR_JOINT_SPHERICAL) {  // log(normalize(q0^-1 q1)), spherical.py:58-62
            const double3 w = dso3_log(dqnormalize(dqmul(dqconj(make_double4(qa[0], qa[1], qa[2], qa[3])),
                                                         make_double4(qb[0], qb[1], qb[2], qb[3]))));
            o[0] = (float)w.x; o[1] = (float)w.y; o[2] = (float)w.z;
          } else {                                // planar.py:70-76, revolute.py:233-237
            const int k = jt == BR_JOINT_PLANAR ? 2 : 0;
            const double dth = atan2((double)qb[k + 1], (double)qb[k]) - atan2((double)qa[k + 1], (double)qa[k]);
            if (jt == BR_JOINT_PLANAR) {
              o[0] = qb[0] - qa[0];
              o[1] = qb[1] - qa[1];
            }
            o[k] = (float)dth;
          }
        }
      }
    }
    __syncwarp();
    // out[e] for the tile's slab: 1:1 slots from the staged inputs, the other slots from above
    float* go = p.out + b0 * lo;
    const int n = cnt * lo;
    auto val = [&](int c, int k) -> float {
      if (!diff) {
        const int kv = vmap[k];
        const float x = A[c * nq + k];
        return kv >= 0 ? x + Bs[c * nv + kv] : x;
      }
      const int kq = qmap[k];
      return kq >= 0 ? Bs[c * nq + kq] - A[c * nq + kq] : A[c * nq - kq - 1];
    };
    int done = 0;
    if (kVec) {
      const int n4 = n >> 2;
      for (int i = lane; i < n4; i += 32) {
        int c = (4 * i) / lo, k = 4 * i - c * lo;
        float r[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          r[u] = val(c, k);
          if (++k == lo) { k = 0; ++c; }
        }
        reinterpret_cast<float4*>(go)[i] = make_float4(r[0], r[1], r[2], r[3]);
      }
      done = n4 << 2;
    }
    for (int e = done + lane; e < n; e += 32) {
      const int c = e / lo;
      go[e] = val(c, e - c * lo);
    }
    __syncwarp();  // this tile's buffer is free for the tiles after the next
  }
  if (kVec) cp_async_wait_all();
}

}  // namespace br

using namespace br;

extern "C" int br_configuration_op(const br_tree_t* tree, const int32_t* active_joints, int32_t n_active, int32_t op,
                                   const float* a, const float* b, int64_t batch, float* out, void* stream) {
  int st = validate_tree(tree);
  if (st) return st;
  if (op != BR_OP_INTEGRATE && op != BR_OP_DIFFERENCE) return BR_EINVAL;
  if (batch < 0 || n_active < 0 || n_active > tree->njoints) return BR_EINVAL;
  if (batch == 0 || n_active == 0) return BR_OK;
  if (!active_joints || !a || !b || !out) return BR_EINVAL;
  if (!aligned4(a) || !aligned4(b) || !aligned4(out)) return BR_EALIGN;
  JointOpParams p = {a, b, out, batch, n_active, op == BR_OP_DIFFERENCE};
  const DeviceInfo& d = device_info();
  const bool vec = aligned16(a) && aligned16(b) && aligned16(out);
  const size_t bytes = (size_t)kJointOpsWarps * joint_ops_warp_floats(tree->nq, tree->nv, p.diff) * sizeof(float);
  if ((int64_t)bytes > d.max_smem_optin) return BR_ETOOBIG;
  auto kern = vec ? joint_ops_kernel<true> : joint_ops_kernel<false>;
  static size_t configured[2][16] = {};
  size_t& have = configured[vec][d.device & 15];
  if (bytes > have) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    have = bytes;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kJointOpsWarps, bytes);
  if (per_sm < 1) per_sm = 1;
  const int64_t tiles = (batch + 31) / 32;
  int64_t blocks = (tiles + kJointOpsWarps - 1) / kJointOpsWarps;
  const int64_t cap = (int64_t)per_sm * d.sms;  // persistent: one wave, then grid-stride over tiles
  if (blocks > cap) blocks = cap;
  kern<<<(unsigned)blocks, 32 * kJointOpsWarps, bytes, (cudaStream_t)stream>>>(*tree, active_joints, p);
  return (int)cudaGetLastError();
}

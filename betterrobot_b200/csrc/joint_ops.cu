// joint_ops.cu — batched configuration-space retraction and difference.
//
// integrate:  q' = q (+) v   (Model.integrate, src/better_robot/data_model/model.py:160-174):
//   revolute / prismatic  q' = q + v                     (revolute.py:46-48)
//   free-flyer            q' = normalize(q * exp(v))     (free_flyer.py:47-51)
// difference: v = q1 (-) q0  (Model.difference, model.py:176-190):
//   revolute / prismatic  v = q1 - q0                    (revolute.py:51-53)
//   free-flyer            v = log(q0^-1 * q1)            (free_flyer.py:53-57)
//
// Layout: a warp owns a tile of 32 consecutive configurations.  Slots of 1:1 joints
// (nq = nv = 1) are processed by the whole warp walking the tile's rows as one
// contiguous range (coalesced loads and stores); free-flyer slots are then processed
// one configuration per lane, so the float64 exp / log runs on all 32 lanes at once
// instead of on one lane of a warp that waits for it.  Memory bound: 4 * (nq + nv + nq)
// bytes per configuration for integrate, 4 * (nq + nq + nv) for difference.
#include <cuda_runtime.h>
#include <stdint.h>

#include "br_common.cuh"
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

__device__ __forceinline__ DPose dpose7(const float* p) {
  return DPose{d3(p[0], p[1], p[2]), make_double4(p[3], p[4], p[5], p[6])};
}

__global__ void __launch_bounds__(256) joint_ops_kernel(const br_tree_t tree, const int32_t* __restrict__ active,
                                                        const JointOpParams p) {
  __shared__ int16_t vmap[BR_MAX_NQ];     // q slot -> v slot of a 1:1 joint, -1 for other slots
  __shared__ int16_t ffq[BR_MAX_JOINTS];  // free-flyer q / v offsets
  __shared__ int16_t ffv[BR_MAX_JOINTS];
  __shared__ int nff;
  const int nq = tree.nq, nv = tree.nv;
  for (int k = threadIdx.x; k < nq; k += blockDim.x) vmap[k] = -1;
  if (threadIdx.x == 0) nff = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < p.n_active; i += blockDim.x) {
    const int j = active[i];
    if (tree.jtype[j] == BR_JOINT_FREE_FLYER) {
      const int s = atomicAdd(&nff, 1);
      ffq[s] = (int16_t)tree.idx_q[j];
      ffv[s] = (int16_t)tree.idx_v[j];
    } else {
      vmap[tree.idx_q[j]] = (int16_t)tree.idx_v[j];
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const int64_t tiles = (p.batch + 31) >> 5;
  const int n_ff = nff;
  for (int64_t tile = (int64_t)blockIdx.x * warps + (threadIdx.x >> 5); tile < tiles;
       tile += (int64_t)gridDim.x * warps) {
    const int64_t b0 = tile << 5;
    const int cnt = p.batch - b0 < 32 ? (int)(p.batch - b0) : 32;
    const int span = cnt * nq;
    const float* a = p.a + b0 * nq;
    if (!p.diff) {
      const float* v = p.b + b0 * nv;
      float* o = p.out + b0 * nq;
      for (int e = lane; e < span; e += 32) {
        const int c = e / nq, k = e - c * nq, kv = vmap[k];
        if (kv >= 0) o[e] = a[e] + v[c * nv + kv];
      }
    } else {
      const float* q1 = p.b + b0 * nq;
      float* o = p.out + b0 * nv;
      for (int e = lane; e < span; e += 32) {
        const int c = e / nq, k = e - c * nq, kv = vmap[k];
        if (kv >= 0) o[c * nv + kv] = q1[e] - a[e];
      }
    }
    if (lane < cnt && n_ff) {
      const int64_t bi = b0 + lane;
      for (int f = 0; f < n_ff; ++f) {
        const int iq = ffq[f], iv = ffv[f];
        const float* qa = p.a + bi * nq + iq;
        if (!p.diff) {
          const float* v = p.b + bi * nv + iv;
          float* o = p.out + bi * nq + iq;
          DPose n = dcompose(dpose7(qa), dse3_exp(d3(v[0], v[1], v[2]), d3(v[3], v[4], v[5])));
          n.q = dqnormalize(n.q);
          o[0] = (float)n.t.x; o[1] = (float)n.t.y; o[2] = (float)n.t.z;
          o[3] = (float)n.q.x; o[4] = (float)n.q.y; o[5] = (float)n.q.z; o[6] = (float)n.q.w;
        } else {
          const float* qb = p.b + bi * nq + iq;
          float* o = p.out + bi * nv + iv;
          double3 v, w;
          dse3_log(dcompose(dinverse(dpose7(qa)), dpose7(qb)), v, w);
          o[0] = (float)v.x; o[1] = (float)v.y; o[2] = (float)v.z;
          o[3] = (float)w.x; o[4] = (float)w.y; o[5] = (float)w.z;
        }
      }
    }
  }
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
  const int threads = 256;
  const int64_t tiles = (batch + 31) / 32;
  int64_t blocks = (tiles + threads / 32 - 1) / (threads / 32);
  const int64_t cap = (int64_t)d.sms * 8;  // 8 CTAs of 256 threads per SM, then grid-stride
  if (blocks > cap) blocks = cap;
  joint_ops_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(*tree, active_joints, p);
  return (int)cudaGetLastError();
}

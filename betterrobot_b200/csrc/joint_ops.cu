// joint_ops.cu — batched configuration-space retraction and difference.
//
// integrate:  q' = q (+) v   (Model.integrate, src/better_robot/data_model/model.py:160-174):
//   revolute / prismatic  q' = q + v                     (revolute.py:46-48)
//   free-flyer            q' = normalize(q * exp(v))     (free_flyer.py:47-51)
// difference: v = q1 (-) q0  (Model.difference, model.py:176-190):
//   revolute / prismatic  v = q1 - q0                    (revolute.py:51-53)
//   free-flyer            v = log(q0^-1 * q1)            (free_flyer.py:53-57)
// One thread per (configuration, joint with nq > 0): consecutive threads touch
// consecutive joints of a configuration, so loads and stores are contiguous.
// Memory bound; computed in float64 and rounded once to float32.
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

__global__ void joint_ops_kernel(const br_tree_t tree, const int32_t* __restrict__ active, const JointOpParams p) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= p.batch * p.n_active) return;
  const int64_t bi = tid / p.n_active;
  const int j = active[tid - bi * p.n_active];
  const int jt = tree.jtype[j], iq = tree.idx_q[j], iv = tree.idx_v[j];
  const int nq = tree.nq, nv = tree.nv;
  const float* a = p.a + bi * nq + iq;
  if (!p.diff) {
    const float* v = p.b + bi * nv + iv;
    float* o = p.out + bi * nq + iq;
    if (jt == BR_JOINT_FREE_FLYER) {
      DPose n = dcompose(dpose7(a), dse3_exp(d3(v[0], v[1], v[2]), d3(v[3], v[4], v[5])));
      n.q = dqnormalize(n.q);
      o[0] = (float)n.t.x; o[1] = (float)n.t.y; o[2] = (float)n.t.z;
      o[3] = (float)n.q.x; o[4] = (float)n.q.y; o[5] = (float)n.q.z; o[6] = (float)n.q.w;
    } else {
      o[0] = (float)((double)a[0] + (double)v[0]);
    }
  } else {
    const float* q1 = p.b + bi * nq + iq;
    float* o = p.out + bi * nv + iv;
    if (jt == BR_JOINT_FREE_FLYER) {
      double3 v, w;
      dse3_log(dcompose(dinverse(dpose7(a)), dpose7(q1)), v, w);
      o[0] = (float)v.x; o[1] = (float)v.y; o[2] = (float)v.z;
      o[3] = (float)w.x; o[4] = (float)w.y; o[5] = (float)w.z;
    } else {
      o[0] = (float)((double)q1[0] - (double)a[0]);
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
  const int64_t n = batch * n_active;
  const int threads = 256;
  const int64_t blocks = (n + threads - 1) / threads;
  if (blocks > 0x7fffffff) return BR_ETOOBIG;
  joint_ops_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(*tree, active_joints, p);
  return (int)cudaGetLastError();
}

// br_fk.cuh — shared-memory pose records and per-joint transforms used by the
// forward-kinematics stages of every kernel in this library.
#pragma once
#include "../../include/br_b200.h"
#include "br_lie.cuh"

namespace br {

__device__ __forceinline__ Pose load_pose8(const float* p) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  const float4 b = *reinterpret_cast<const float4*>(p + 4);
  Pose T;
  T.t = f3(a.x, a.y, a.z);
  T.q = b;
  return T;
}
__device__ __forceinline__ void store_pose8(float* p, const Pose& T) {
  *reinterpret_cast<float4*>(p) = make_float4(T.t.x, T.t.y, T.t.z, 0.f);
  *reinterpret_cast<float4*>(p + 4) = T.q;
}
__device__ __forceinline__ Pose load_split(const float* pt, const float* pq, int j) {
  const float4 a = *reinterpret_cast<const float4*>(pt + 4 * j);
  Pose T;
  T.t = f3(a.x, a.y, a.z);
  T.q = *reinterpret_cast<const float4*>(pq + 4 * j);
  return T;
}
__device__ __forceinline__ void store_split(float* pt, float* pq, int j, const Pose& T) {
  *reinterpret_cast<float4*>(pt + 4 * j) = make_float4(T.t.x, T.t.y, T.t.z, 0.f);
  *reinterpret_cast<float4*>(pq + 4 * j) = T.q;
}
__device__ __forceinline__ void store_pose7(float* p, const Pose& T) {
  p[0] = T.t.x; p[1] = T.t.y; p[2] = T.t.z;
  p[3] = T.q.x; p[4] = T.q.y; p[5] = T.q.z; p[6] = T.q.w;
}

// liMi_j = placement_j * T_j(q_j)   (forward.py:114-122; joint_transform of
// revolute.py:18-21, prismatic.py:16-19, free_flyer.py:31-36, fixed.py:90-94)
__device__ __forceinline__ Pose local_transform(int jt, const Pose& P, const float* __restrict__ axis4,
                                                const float* __restrict__ qv) {
  Pose L = P;
  if (jt == BR_JOINT_REVOLUTE) {
    float s, c;
    sincosf(0.5f * qv[0], &s, &c);
    const float4 qj = make_float4(s * axis4[0], s * axis4[1], s * axis4[2], c);
    L.q = qmul(P.q, qj);
  } else if (jt == BR_JOINT_PRISMATIC) {
    const float d = qv[0];
    L.t = add(P.t, qrot(P.q, f3(d * axis4[0], d * axis4[1], d * axis4[2])));
  } else if (jt == BR_JOINT_FREE_FLYER) {
    Pose F;
    F.t = f3(qv[0], qv[1], qv[2]);
    F.q = qnormalize(make_float4(qv[3], qv[4], qv[5], qv[6]));
    L = compose(P, F);
  }
  return L;
}

}  // namespace br

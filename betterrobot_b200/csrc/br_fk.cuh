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

// Degrees of freedom (tangent columns) of a joint kind.
__host__ __device__ __forceinline__ int joint_nv(int jt) {
  switch (jt) {
    case BR_JOINT_REVOLUTE: case BR_JOINT_PRISMATIC: case BR_JOINT_REVOLUTE_UNBOUNDED: return 1;
    case BR_JOINT_SPHERICAL: case BR_JOINT_PLANAR: case BR_JOINT_TRANSLATION: return 3;
    case BR_JOINT_FREE_FLYER: return 6;
    default: return 0;
  }
}
__host__ __device__ __forceinline__ int joint_nq(int jt) {
  switch (jt) {
    case BR_JOINT_REVOLUTE: case BR_JOINT_PRISMATIC: return 1;
    case BR_JOINT_REVOLUTE_UNBOUNDED: return 2;
    case BR_JOINT_TRANSLATION: return 3;
    case BR_JOINT_SPHERICAL: case BR_JOINT_PLANAR: return 4;
    case BR_JOINT_FREE_FLYER: return 7;
    default: return 0;
  }
}
// Kinds whose configuration slots are their tangent coordinates (q + v, nq == nv).
__host__ __device__ __forceinline__ bool joint_is_vector(int jt) {
  return jt == BR_JOINT_REVOLUTE || jt == BR_JOINT_PRISMATIC || jt == BR_JOINT_TRANSLATION;
}
// Planar rotation quaternion from (cos, sin): half angles from cos, sign from sin, as
// planar.py:31-33 computes them (sign(0) = 0).
__device__ __forceinline__ float4 planar_quat(float c, float s) {
  const float hc = sqrtf(fmaxf(0.5f * (1.f + c), 0.f));
  const float hs = sqrtf(fmaxf(0.5f * (1.f - c), 0.f)) * (float)((s > 0.f) - (s < 0.f));
  return make_float4(0.f, 0.f, hs, hc);
}
__device__ __forceinline__ double4 dplanar_quat(double c, double s) {
  const double hc = sqrt(fmax(0.5 * (1.0 + c), 0.0));
  const double hs = sqrt(fmax(0.5 * (1.0 - c), 0.0)) * (double)((s > 0.0) - (s < 0.0));
  return make_double4(0.0, 0.0, hs, hc);
}

// liMi_j = placement_j * T_j(q_j)   (forward.py:114-122; joint_transform of
// revolute.py:18-21 and :206-211, prismatic.py:16-19, free_flyer.py:31-36,
// spherical.py:22-32, planar.py:20-41, translation.py:19-23, fixed.py:90-94)
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
  } else if (jt == BR_JOINT_SPHERICAL) {
    L.q = qmul(P.q, qnormalize(make_float4(qv[0], qv[1], qv[2], qv[3])));
  } else if (jt == BR_JOINT_PLANAR) {
    L.t = add(P.t, qrot(P.q, f3(qv[0], qv[1], 0.f)));
    L.q = qmul(P.q, planar_quat(qv[2], qv[3]));
  } else if (jt == BR_JOINT_REVOLUTE_UNBOUNDED) {
    float s, c;
    sincosf(0.5f * atan2f(qv[1], qv[0]), &s, &c);
    L.q = qmul(P.q, make_float4(s * axis4[0], s * axis4[1], s * axis4[2], c));
  } else if (jt == BR_JOINT_TRANSLATION) {
    L.t = add(P.t, qrot(P.q, f3(qv[0], qv[1], qv[2])));
  }
  return L;
}

// float64 liMi_j for the LM / trajectory kernels (same cases as local_transform).  With
// kAllKinds = false only fixed, revolute, prismatic and free-flyer joints are compiled in.
template <bool kAllKinds = true>
__device__ __forceinline__ DPose dlocal_transform(int jt, const DPose& P, const float* __restrict__ axis4,
                                                  const double* __restrict__ qv) {
  DPose L = P;
  if (jt == BR_JOINT_REVOLUTE || (kAllKinds && jt == BR_JOINT_REVOLUTE_UNBOUNDED)) {
    const double th = jt == BR_JOINT_REVOLUTE ? qv[0] : atan2(qv[1], qv[0]);
    double s, c;
    sincospi(th * (0.5 / 3.141592653589793), &s, &c);  // sin, cos of th / 2 (no large-argument reduction path)
    L.q = dqmul(P.q, make_double4(s * axis4[0], s * axis4[1], s * axis4[2], c));
  } else if (jt == BR_JOINT_PRISMATIC) {
    L.t = dadd(P.t, dqrot(P.q, d3(qv[0] * axis4[0], qv[0] * axis4[1], qv[0] * axis4[2])));
  } else if (jt == BR_JOINT_FREE_FLYER) {
    L = dcompose(P, DPose{d3(qv[0], qv[1], qv[2]), dqnormalize(make_double4(qv[3], qv[4], qv[5], qv[6]))});
  } else if (kAllKinds && jt == BR_JOINT_SPHERICAL) {
    L.q = dqmul(P.q, dqnormalize(make_double4(qv[0], qv[1], qv[2], qv[3])));
  } else if (kAllKinds && jt == BR_JOINT_PLANAR) {
    L.t = dadd(P.t, dqrot(P.q, d3(qv[0], qv[1], 0.0)));
    L.q = dqmul(P.q, dplanar_quat(qv[2], qv[3]));
  } else if (kAllKinds && jt == BR_JOINT_TRANSLATION) {
    L.t = dadd(P.t, dqrot(P.q, d3(qv[0], qv[1], qv[2])));
  }
  return L;
}

// Joint kinds the plain LM variant is compiled for (bit BR_JOINT_k).
constexpr int kBasicKinds = (1 << BR_JOINT_FIXED) | (1 << BR_JOINT_REVOLUTE) | (1 << BR_JOINT_PRISMATIC) |
                            (1 << BR_JOINT_FREE_FLYER);

}  // namespace br

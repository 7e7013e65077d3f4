// lie_ops.cu — batched SE3 / SO3 primitives: the per-op LieOps seam of
// src/better_robot/backends/protocol.py:27-51, with the semantics of
// src/better_robot/lie/_torch_native_backend.py (storage [tx,ty,tz,qx,qy,qz,qw],
// tangents [v, w], linear first) and the SE3 right Jacobians of
// src/better_robot/lie/tangents.py:184-207.
//
// One lane per element, one warp per tile of 32 consecutive elements (grid-stride over
// tiles), one kernel instantiation per op.  The same device functions run inside the
// fused FK / Jacobian / LM / adjoint kernels, so this entry point also exposes them to
// parity tests one operation at a time.  Records are 3..36 floats; a tile's records are
// contiguous slabs, staged through shared memory by cp.async on the way in and written
// back with coalesced 16-byte stores (lie_ops_kernel below).
#include <cuda_runtime.h>
#include <stdint.h>

#include "br_common.cuh"
#include "br_lie.cuh"

namespace br {

struct LieOpSpec {
  int8_t a, b, out;  // floats per element of a, b (0: unused), out
};

// Indexed by BR_LIE_* (include/br_b200.h).
__host__ __device__ constexpr LieOpSpec lie_spec(int op) {
  switch (op) {
    case BR_LIE_SE3_COMPOSE: return {7, 7, 7};
    case BR_LIE_SE3_INVERSE: return {7, 0, 7};
    case BR_LIE_SE3_LOG: return {7, 0, 6};
    case BR_LIE_SE3_EXP: return {6, 0, 7};
    case BR_LIE_SE3_ACT: return {7, 3, 3};
    case BR_LIE_SE3_ADJOINT: return {7, 0, 36};
    case BR_LIE_SE3_ADJOINT_INV: return {7, 0, 36};
    case BR_LIE_SE3_NORMALIZE: return {7, 0, 7};
    case BR_LIE_SO3_COMPOSE: return {4, 4, 4};
    case BR_LIE_SO3_INVERSE: return {4, 0, 4};
    case BR_LIE_SO3_LOG: return {4, 0, 3};
    case BR_LIE_SO3_EXP: return {3, 0, 4};
    case BR_LIE_SO3_ACT: return {4, 3, 3};
    case BR_LIE_SO3_TO_MATRIX: return {4, 0, 9};
    case BR_LIE_SO3_FROM_MATRIX: return {9, 0, 4};
    case BR_LIE_SO3_NORMALIZE: return {4, 0, 4};
    case BR_LIE_SE3_JR: return {6, 0, 36};
    case BR_LIE_SE3_JR_INV: return {6, 0, 36};
    default: return {0, 0, 0};
  }
}

__device__ __forceinline__ Pose ld_pose(const float* p) {
  Pose P;
  P.t = f3(p[0], p[1], p[2]);
  P.q = make_float4(p[3], p[4], p[5], p[6]);
  return P;
}
__device__ __forceinline__ void st_pose(float* o, const Pose& P) {
  o[0] = P.t.x; o[1] = P.t.y; o[2] = P.t.z;
  o[3] = P.q.x; o[4] = P.q.y; o[5] = P.q.z; o[6] = P.q.w;
}
__device__ __forceinline__ float4 ld_quat(const float* p) { return make_float4(p[0], p[1], p[2], p[3]); }
__device__ __forceinline__ void st_quat(float* o, float4 q) { o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w; }
__device__ __forceinline__ void st3(float* o, float3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

// Row-major 3x3 rotation of a unit quaternion (_quat_to_matrix, _torch_native_backend.py:55-69).
__device__ __forceinline__ void quat_to_matrix(float4 q, float* R) {
  const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
  const float xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
  const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
  R[0] = 1.f - 2.f * (yy + zz); R[1] = 2.f * (xy - wz);        R[2] = 2.f * (xz + wy);
  R[3] = 2.f * (xy + wz);       R[4] = 1.f - 2.f * (xx + zz);  R[5] = 2.f * (yz - wx);
  R[6] = 2.f * (xz - wy);       R[7] = 2.f * (yz + wx);        R[8] = 1.f - 2.f * (xx + yy);
}

// Shepperd's method with the reference's branch order and clamps
// (_matrix_to_quat, _torch_native_backend.py:72-125), then normalised.
__device__ __forceinline__ float4 matrix_to_quat(const float* m) {
  const float tr = m[0] + m[4] + m[8];
  float4 q;
  if (tr > 0.f) {
    const float s = sqrtf(fmaxf(tr + 1.f, 1e-30f)) * 2.f;
    q = make_float4((m[7] - m[5]) / s, (m[2] - m[6]) / s, (m[3] - m[1]) / s, 0.25f * s);
  } else if (m[0] > m[4] && m[0] > m[8]) {
    const float s = sqrtf(fmaxf(1.f + m[0] - m[4] - m[8], 1e-30f)) * 2.f;
    q = make_float4(0.25f * s, (m[1] + m[3]) / s, (m[2] + m[6]) / s, (m[7] - m[5]) / s);
  } else if (m[4] > m[8]) {
    const float s = sqrtf(fmaxf(1.f - m[0] + m[4] - m[8], 1e-30f)) * 2.f;
    q = make_float4((m[1] + m[3]) / s, 0.25f * s, (m[5] + m[7]) / s, (m[2] - m[6]) / s);
  } else {
    const float s = sqrtf(fmaxf(1.f - m[0] - m[4] + m[8], 1e-30f)) * 2.f;
    q = make_float4((m[2] + m[6]) / s, (m[5] + m[7]) / s, 0.25f * s, (m[3] - m[1]) / s);
  }
  const float n = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-12f);
  return make_float4(q.x / n, q.y / n, q.z / n, q.w / n);
}

// Ad(T) = [[R, hat(p) R], [0, R]]; Ad(T^-1) = [[R^T, -R^T hat(p)], [0, R^T]]
// (se3_adjoint / se3_adjoint_inv, _torch_native_backend.py:318-342), row-major 6x6.
__device__ __forceinline__ void se3_adjoint_rows(const Pose& T, bool inv, float* o) {
  float R[9];
  quat_to_matrix(T.q, R);
  const float3 p = T.t;
  // hat(p) rows: [0,-pz,py], [pz,0,-px], [-py,px,0]
  const float H[9] = {0.f, -p.z, p.y, p.z, 0.f, -p.x, -p.y, p.x, 0.f};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float r = inv ? R[j * 3 + i] : R[i * 3 + j];
      float x = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) x += inv ? -R[k * 3 + i] * H[k * 3 + j] : H[i * 3 + k] * R[k * 3 + j];
      o[i * 6 + j] = r;
      o[i * 6 + 3 + j] = x;
      o[(i + 3) * 6 + j] = 0.f;
      o[(i + 3) * 6 + 3 + j] = r;
    }
  }
}

// Jr(xi) = sum_{k=0}^{9} (-1)^k/(k+1)! ad(xi)^k, ad = [[W, V], [0, W]]
// (tangents.right_jacobian_se3:184-201, tangents._ad_matrix:164-178), evaluated by
// Horner's rule on the 6x6 matrix: Jr = c0 I + ad(c1 I + ad(c2 I + ... )).
__device__ __forceinline__ void se3_jr_rows(float3 v, float3 w, float* o) {
  float ad[36];
  const float W[9] = {0.f, -w.z, w.y, w.z, 0.f, -w.x, -w.y, w.x, 0.f};
  const float V[9] = {0.f, -v.z, v.y, v.z, 0.f, -v.x, -v.y, v.x, 0.f};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      ad[i * 6 + j] = W[i * 3 + j];
      ad[i * 6 + 3 + j] = V[i * 3 + j];
      ad[(i + 3) * 6 + j] = 0.f;
      ad[(i + 3) * 6 + 3 + j] = W[i * 3 + j];
    }
  }
  // coefficients (-1)^k / (k+1)!, k = 0..9
  const float c[10] = {1.f, -1.f / 2.f, 1.f / 6.f, -1.f / 24.f, 1.f / 120.f, -1.f / 720.f, 1.f / 5040.f,
                       -1.f / 40320.f, 1.f / 362880.f, -1.f / 3628800.f};
  float acc[36], tmp[36];
#pragma unroll
  for (int e = 0; e < 36; ++e) acc[e] = (e % 7 == 0) ? c[9] : 0.f;
  for (int k = 8; k >= 0; --k) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        float x = (i == j) ? c[k] : 0.f;
#pragma unroll
        for (int l = 0; l < 6; ++l) x = fmaf(ad[i * 6 + l], acc[l * 6 + j], x);
        tmp[i * 6 + j] = x;
      }
    }
#pragma unroll
    for (int e = 0; e < 36; ++e) acc[e] = tmp[e];
  }
#pragma unroll
  for (int e = 0; e < 36; ++e) o[e] = acc[e];
}

template <int OP>
__device__ __forceinline__ void apply_op(const float* x, const float* y, float* o) {
  if constexpr (OP == BR_LIE_SE3_COMPOSE) {
    st_pose(o, compose(ld_pose(x), ld_pose(y)));
  } else if constexpr (OP == BR_LIE_SE3_INVERSE) {
    st_pose(o, inverse(ld_pose(x)));
  } else if constexpr (OP == BR_LIE_SE3_LOG) {
    float3 v, w;
    se3_log(ld_pose(x), v, w);
    st3(o, v);
    st3(o + 3, w);
  } else if constexpr (OP == BR_LIE_SE3_EXP) {
    st_pose(o, se3_exp(f3(x[0], x[1], x[2]), f3(x[3], x[4], x[5])));
  } else if constexpr (OP == BR_LIE_SE3_ACT) {
    const Pose T = ld_pose(x);
    st3(o, add(qrot(T.q, f3(y[0], y[1], y[2])), T.t));
  } else if constexpr (OP == BR_LIE_SE3_ADJOINT) {
    se3_adjoint_rows(ld_pose(x), false, o);
  } else if constexpr (OP == BR_LIE_SE3_ADJOINT_INV) {
    se3_adjoint_rows(ld_pose(x), true, o);
  } else if constexpr (OP == BR_LIE_SE3_NORMALIZE) {
    Pose T = ld_pose(x);
    T.q = qnormalize(T.q);
    st_pose(o, T);
  } else if constexpr (OP == BR_LIE_SO3_COMPOSE) {
    st_quat(o, qmul(ld_quat(x), ld_quat(y)));
  } else if constexpr (OP == BR_LIE_SO3_INVERSE) {
    st_quat(o, qconj(ld_quat(x)));
  } else if constexpr (OP == BR_LIE_SO3_LOG) {
    st3(o, so3_log(ld_quat(x)));
  } else if constexpr (OP == BR_LIE_SO3_EXP) {
    st_quat(o, so3_exp(f3(x[0], x[1], x[2])));
  } else if constexpr (OP == BR_LIE_SO3_ACT) {
    st3(o, qrot(ld_quat(x), f3(y[0], y[1], y[2])));
  } else if constexpr (OP == BR_LIE_SO3_TO_MATRIX) {
    quat_to_matrix(ld_quat(x), o);
  } else if constexpr (OP == BR_LIE_SO3_FROM_MATRIX) {
    float m[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = x[e];
    st_quat(o, matrix_to_quat(m));
  } else if constexpr (OP == BR_LIE_SO3_NORMALIZE) {
    st_quat(o, qnormalize(ld_quat(x)));
  } else if constexpr (OP == BR_LIE_SE3_JR) {
    se3_jr_rows(f3(x[0], x[1], x[2]), f3(x[3], x[4], x[5]), o);
  } else if constexpr (OP == BR_LIE_SE3_JR_INV) {
    const JrInv J = jr_inv_se3<9>(f3(x[0], x[1], x[2]), f3(x[3], x[4], x[5]));
    // column c of Jr^-1 = Jr^-1 e_c
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      float3 ol, oa;
      jr_inv_apply(J, f3(c == 0, c == 1, c == 2), f3(c == 3, c == 4, c == 5), ol, oa);
      o[0 * 6 + c] = ol.x; o[1 * 6 + c] = ol.y; o[2 * 6 + c] = ol.z;
      o[3 * 6 + c] = oa.x; o[4 * 6 + c] = oa.y; o[5 * 6 + c] = oa.z;
    }
  }
}

// Start copying `len` floats of a global slab into a warp's shared-memory tile without passing
// through registers: 16-byte cp.async while both sides allow it (`vec`: the slab starts on a
// 16-byte boundary; tiles start on one), then 4-byte copies for the remainder.  The caller
// commits the group and waits for it.
__device__ __forceinline__ void warp_load_async(float* __restrict__ s, const float* __restrict__ g, int len,
                                                int lane, bool vec) {
  int k0 = 0;
  if (vec) {
    const int n4 = len >> 2;
    for (int k = lane; k < n4; k += kWarp) cp_async16(s + 4 * k, g + 4 * k);
    k0 = n4 << 2;
  }
  for (int k = k0 + lane; k < len; k += kWarp) cp_async4(s + k, g + k);
}
// Copy `len` floats of a warp's output tile to global memory, coalesced (16-byte stores while
// the destination allows them).
__device__ __forceinline__ void warp_store(float* __restrict__ g, const float* __restrict__ s, int len, int lane,
                                           bool vec) {
  int k0 = 0;
  if (vec) {
    const int n4 = len >> 2;
    for (int k = lane; k < n4; k += kWarp) reinterpret_cast<float4*>(g)[k] = reinterpret_cast<const float4*>(s)[k];
    k0 = n4 << 2;
  }
  for (int k = k0 + lane; k < len; k += kWarp) g[k] = s[k];
}

constexpr int kLieWarps = 8;  // warps per CTA

// One warp per tile of 32 consecutive elements: the tile's operand records (contiguous slabs
// of 32 * floats-per-record) are copied into the warp's shared memory by cp.async, the NEXT
// tile's into a second buffer while this one is computed where shared memory allows (so a
// warp keeps a whole tile of loads in flight), each lane applies the op to its element, and the output slab leaves with
// coalesced stores.  A broadcast operand (one record for every element) is read in place.
template <int OP>
__global__ void __launch_bounds__(kLieWarps * kWarp) lie_ops_kernel(const float* __restrict__ a,
                                                                   const float* __restrict__ b, int64_t n,
                                                                   int a_bcast, int b_bcast, float* __restrict__ out) {
  constexpr LieOpSpec sp = lie_spec(OP);
  constexpr int A = sp.a, Bn = sp.b, O = sp.out;
  constexpr int IN = kWarp * (A + Bn);         // input floats per tile (a multiple of 4: 16-byte tiles)
  // two input buffers and the output tile per warp, while the CTA's static shared memory allows
  // (the 36-float outputs of the adjoint and Jr ops leave room for one input buffer only)
  constexpr int NB = kLieWarps * (2 * IN + kWarp * O) * 4 <= 48 * 1024 ? 2 : 1;
  constexpr int TILE = NB * IN + kWarp * O;
  __shared__ __align__(16) float smem[kLieWarps * TILE];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float* sbuf = smem + w * TILE;
  float* so = sbuf + NB * IN;                  // the output tile follows the NB input buffers
  static_assert(NB * IN + kWarp * O == TILE, "a warp's input buffers and output tile fill its slice");
  const bool va = ((reinterpret_cast<uintptr_t>(a) & 15u) == 0), vb = ((reinterpret_cast<uintptr_t>(b) & 15u) == 0),
             vo = ((reinterpret_cast<uintptr_t>(out) & 15u) == 0);
  const int64_t ntiles = (n + kWarp - 1) / kWarp;
  const int64_t step = (int64_t)gridDim.x * kLieWarps;
  auto fetch = [&](int64_t t, float* buf) {  // issue tile t's operand copies into buf
    const int64_t i0 = t * kWarp;
    const int cnt = (int)((n - i0) < kWarp ? (n - i0) : kWarp);
    if (!a_bcast) warp_load_async(buf, a + i0 * A, cnt * A, lane, va);
    if (Bn && !b_bcast) warp_load_async(buf + kWarp * A, b + i0 * Bn, cnt * Bn, lane, vb);
  };
  int64_t t = (int64_t)blockIdx.x * kLieWarps + w;
  if (NB == 2 && t < ntiles) fetch(t, sbuf);
  cp_async_commit();
  for (int k = 0; t < ntiles; t += step, ++k) {
    float* cur = sbuf + (NB == 2 ? (k & 1) * IN : 0);
    if (NB == 1) fetch(t, cur);
    else if (t + step < ntiles) fetch(t + step, sbuf + ((k + 1) & 1) * IN);
    cp_async_commit();
    if (NB == 2) cp_async_wait_groups<1>();    // this tile's copies are done (the next one's may fly)
    else cp_async_wait_groups<0>();
    __syncwarp();
    const int64_t i0 = t * kWarp;
    const int cnt = (int)((n - i0) < kWarp ? (n - i0) : kWarp);
    if (lane < cnt) {
      const float* x = a_bcast ? a : cur + lane * A;
      const float* y = Bn ? (b_bcast ? b : cur + kWarp * A + lane * Bn) : nullptr;
      apply_op<OP>(x, y, so + lane * O);
    }
    __syncwarp();
    warp_store(out + i0 * O, so, cnt * O, lane, vo);
    __syncwarp();                              // cur and so are free for the next tiles
  }
  cp_async_wait_all();
}

template <int OP>
static void launch_op(unsigned blocks, cudaStream_t s, const float* a, const float* b, int64_t n, int ab, int bb,
                      float* out) {
  lie_ops_kernel<OP><<<blocks, kLieWarps * kWarp, 0, s>>>(a, b, n, ab, bb, out);
}

}  // namespace br

using namespace br;

extern "C" int br_lie_op_sizes(int32_t op, int32_t* a_floats, int32_t* b_floats, int32_t* out_floats) {
  const LieOpSpec sp = lie_spec(op);
  if (sp.out == 0) return BR_EINVAL;
  if (a_floats) *a_floats = sp.a;
  if (b_floats) *b_floats = sp.b;
  if (out_floats) *out_floats = sp.out;
  return BR_OK;
}

extern "C" int br_lie_op(int32_t op, const float* a, int64_t na, const float* b, int64_t nb, float* out, int64_t n,
                         void* stream) {
  const LieOpSpec sp = lie_spec(op);
  if (sp.out == 0 || n < 0) return BR_EINVAL;
  if (n == 0) return BR_OK;
  if (!a || !out || (na != n && na != 1)) return BR_EINVAL;
  if (sp.b && (!b || (nb != n && nb != 1))) return BR_EINVAL;
  if (!aligned4(a) || !aligned4(out) || (sp.b && !aligned4(b))) return BR_EALIGN;
  const DeviceInfo& d = device_info();
  int64_t blocks = (n + kLieWarps * kWarp - 1) / (kLieWarps * kWarp);   // one 32-element tile per warp
  const int64_t cap = (int64_t)d.sms * 8;  // grid-stride beyond 8 CTAs of 8 warps per SM (64 warps: the SM's limit)
  if (blocks > cap) blocks = cap;
  const cudaStream_t s = (cudaStream_t)stream;
  const unsigned g = (unsigned)blocks;
  const float* bp = sp.b ? b : nullptr;
  const int ab = na == 1, bb = nb == 1;
  switch (op) {
#define BR_LIE_CASE(OP) \
  case OP: launch_op<OP>(g, s, a, bp, n, ab, bb, out); break;
    BR_LIE_CASE(BR_LIE_SE3_COMPOSE) BR_LIE_CASE(BR_LIE_SE3_INVERSE) BR_LIE_CASE(BR_LIE_SE3_LOG)
    BR_LIE_CASE(BR_LIE_SE3_EXP) BR_LIE_CASE(BR_LIE_SE3_ACT) BR_LIE_CASE(BR_LIE_SE3_ADJOINT)
    BR_LIE_CASE(BR_LIE_SE3_ADJOINT_INV) BR_LIE_CASE(BR_LIE_SE3_NORMALIZE) BR_LIE_CASE(BR_LIE_SO3_COMPOSE)
    BR_LIE_CASE(BR_LIE_SO3_INVERSE) BR_LIE_CASE(BR_LIE_SO3_LOG) BR_LIE_CASE(BR_LIE_SO3_EXP)
    BR_LIE_CASE(BR_LIE_SO3_ACT) BR_LIE_CASE(BR_LIE_SO3_TO_MATRIX) BR_LIE_CASE(BR_LIE_SO3_FROM_MATRIX)
    BR_LIE_CASE(BR_LIE_SO3_NORMALIZE) BR_LIE_CASE(BR_LIE_SE3_JR) BR_LIE_CASE(BR_LIE_SE3_JR_INV)
#undef BR_LIE_CASE
    default: return BR_EINVAL;
  }
  return (int)cudaGetLastError();
}

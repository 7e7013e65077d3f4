// br_lie.cuh — SE3 / SO3 device functions (float32).
//
// Same conventions and formulas as BetterRobot's torch backend
// (src/better_robot/lie/_torch_native_backend.py): poses [t, q] with scalar-last
// quaternions, tangents [v, w] linear first.  Where a float64 formula loses
// precision in float32 (1 - cos, theta - sin, 1/theta^2 - cot(theta/2)/(2 theta))
// the coefficient is evaluated from its Taylor series below a cutoff instead, so
// results agree with the float64 reference to float32 rounding.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace br {

struct Pose {
  float3 t;
  float4 q;  // (x, y, z, w)
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 scale(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return f3(fmaf(a.y, b.z, -a.z * b.y), fmaf(a.z, b.x, -a.x * b.z), fmaf(a.x, b.y, -a.y * b.x));
}
// a + s * b
__device__ __forceinline__ float3 axpy(float s, float3 b, float3 a) {
  return f3(fmaf(s, b.x, a.x), fmaf(s, b.y, a.y), fmaf(s, b.z, a.z));
}

// Hamilton product a (x) b   (_quat_mul, _torch_native_backend.py:44-52)
__device__ __forceinline__ float4 qmul(float4 a, float4 b) {
  float4 r;
  r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  r.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
  r.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
  r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  return r;
}

__device__ __forceinline__ float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }

// p' = p + 2 u x (u x p + w p)   (so3_act, _torch_native_backend.py:186-199)
__device__ __forceinline__ float3 qrot(float4 q, float3 p) {
  const float3 u = f3(q.x, q.y, q.z);
  const float3 c1 = axpy(q.w, p, cross(u, p));
  return axpy(2.f, cross(u, c1), p);
}
__device__ __forceinline__ float3 qrot_inv(float4 q, float3 p) { return qrot(qconj(q), p); }

// c = a * b   (se3_compose, _torch_native_backend.py:237-246)
__device__ __forceinline__ Pose compose(const Pose& a, const Pose& b) {
  Pose c;
  c.t = add(a.t, qrot(a.q, b.t));
  c.q = qmul(a.q, b.q);
  return c;
}

// T^-1   (se3_inverse, _torch_native_backend.py:249-255)
__device__ __forceinline__ Pose inverse(const Pose& a) {
  Pose r;
  r.q = qconj(a.q);
  r.t = scale(qrot(r.q, a.t), -1.f);
  return r;
}

// (se3_normalize, _torch_native_backend.py:358-361): quaternion / max(|q|, 1e-8)
__device__ __forceinline__ float4 qnormalize(float4 q) {
  const float n = fmaxf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w), 1e-8f);
  const float s = 1.f / n;
  return make_float4(q.x * s, q.y * s, q.z * s, q.w * s);
}

// theta / sin(theta/2) factor of so3_log and the log itself
// (so3_log, _torch_native_backend.py:162-183; folds qw < 0 onto the same rotation).
__device__ __forceinline__ float3 so3_log(float4 q) {
  if (q.w < 0.f) q = make_float4(-q.x, -q.y, -q.z, -q.w);
  const float s2 = q.x * q.x + q.y * q.y + q.z * q.z;
  const float s = sqrtf(s2);
  float factor;
  if (s2 < 0.25e-8f) {
    factor = 2.f + s2 * (2.f / 3.f);
  } else {
    const float theta = 2.f * atan2f(s, fminf(fmaxf(q.w, -1.f), 1.f));
    factor = theta / s;
  }
  return f3(factor * q.x, factor * q.y, factor * q.z);
}

// c(theta) = 1/theta^2 - cot(theta/2) / (2 theta), the W^2 coefficient of V^-1
// (se3_log, _torch_native_backend.py:298-303) and of the SO3 Jr^-1
// (tangents.right_jacobian_inv_so3:122-145).  Series 1/12 + t2/720 + t2^2/30240
// + t2^3/1209600 + t2^4/47900160 below theta = 1 (float32 cancels there).
__device__ __forceinline__ float vinv_series(float th2) {
  return fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 47900160.f, 1.f / 1209600.f), 1.f / 30240.f), 1.f / 720.f),
              1.f / 12.f);
}
__device__ __forceinline__ float vinv_coeff(float th2) {
  if (th2 < 1.f) return vinv_series(th2);
  const float th = sqrtf(th2);
  float sh, ch;
  sincospif(th * (0.5f / 3.14159265358979f), &sh, &ch);  // sin, cos of th / 2 (th <= pi for a log)
  return 1.f / th2 - (ch / sh) / (2.f * th);
}

// Jr^-1(xi)^T xi for xi = (v, w): the gradient of 1/2 |log(T0^-1 T)|^2 with respect to a
// right perturbation of T, in closed form.  With Jr(xi) = [[A, B], [0, A]] (A = Jr_so3(w)),
// A^-T = Jl_so3(w)^-1 = V(w)^-1 and A^-T w = w, B^T = Q_l(v, w) (the left-Jacobian block of
// Barfoot, "State Estimation for Robotics", eq. 7.86b), so
//   g_lin = V^-1 v,   g_ang = w - V^-1 Q_l(v, w) g_lin
// with Q_l u = 1/2 v x u + c2 (w^v^ + v^w^ + w^v^w^) u + c3 (w^w^v^ + v^w^w^ - 3 w^v^w^) u
//             + c4 (w^v^w^w^ + w^w^v^w^) u,
// c2 = (th - sin th)/th^3, c3 = (th^2 + 2 cos th - 2)/(2 th^4), c4 = (2 th - 3 sin th + th cos th)/(2 th^5)
// (Taylor series of each for th^2 < 2, where the closed forms cancel).  Equal to applying the
// exact (infinite-series) Jr^-1 of jr_inv_se3 below, at a fraction of its arithmetic.  Beyond
// th = 1 one sincos of th/2 and one reciprocal r = 1/(th sin(th/2)) give every coefficient:
// sin th = 2 sin(th/2) cos(th/2), cos th = 1 - 2 sin^2(th/2), 1/th = sin(th/2) r,
// cot(th/2) = th cos(th/2) r.
__device__ __forceinline__ void jr_inv_T_xi(float3 v, float3 w, float3& gl, float3& ga) {
  const float th2 = dot(w, w);
  float c, c2, c3, c4;
  if (th2 < 2.f) {
    c2 = fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 39916800.f, -1.f / 362880.f), 1.f / 5040.f), -1.f / 120.f),
              1.f / 6.f);
    c3 = fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 479001600.f, -1.f / 3628800.f), 1.f / 40320.f),
                   -1.f / 720.f), 1.f / 24.f);
    c4 = fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 1245404160.f, -1.f / 9979200.f), 1.f / 120960.f),
                   -1.f / 2520.f), 1.f / 120.f);
  }
  if (th2 < 1.f) {
    c = vinv_series(th2);
  } else {
    const float th = sqrtf(th2);
    float sh, ch;
    sincospif(th * (0.5f / 3.14159265358979f), &sh, &ch);
    const float r = 1.f / (th * sh);
    const float it = sh * r;                       // 1 / th
    c = it * fmaf(-0.5f * ch, th * r, it);         // 1/th^2 - cot(th/2) / (2 th)
    if (th2 >= 2.f) {
      const float s = 2.f * sh * ch, co = fmaf(-2.f * sh, sh, 1.f);
      const float it2 = it * it;
      c2 = (th - s) * (it2 * it);
      c3 = 0.5f * (th2 + 2.f * co - 2.f) * (it2 * it2);
      c4 = 0.5f * (2.f * th - 3.f * s + th * co) * (it2 * it2 * it);
    }
  }
  auto vinv = [&](float3 x) { return axpy(c, cross(w, cross(w, x)), axpy(-0.5f, cross(w, x), x)); };
  gl = vinv(v);
  const float3 a1 = cross(w, gl), a2 = cross(w, a1);
  const float3 b0 = cross(v, gl), b1 = cross(v, a1), b2 = cross(v, a2);
  const float3 wb0 = cross(w, b0), wwb0 = cross(w, wb0), wb1 = cross(w, b1), wwb1 = cross(w, wb1);
  const float3 wb2 = cross(w, b2);
  float3 q = scale(b0, 0.5f);
  q = axpy(c2, add(add(wb0, b1), wb1), q);
  q = axpy(c3, add(add(wwb0, b2), scale(wb1, -3.f)), q);
  q = axpy(c4, add(wb2, wwb1), q);
  ga = sub(w, vinv(q));
}

// atan2(y, x) for y, x >= 0, not both 0 (the first quadrant, where the logs need it):
// atan(r) = r P(r^2) on r = min / max in [0, 1], reflected as pi/2 - atan(r) when y > x.
// P is a degree-8 polynomial fitted here to atan(r) / r by least squares on Chebyshev-spaced
// points of [0, 1], iteratively reweighted towards the minimax error: 5.8e-9 rad in exact
// arithmetic, 9.2e-8 rad (2 ulp at pi/4) evaluated in float32 by Horner's rule.
__device__ __forceinline__ float atan_q1(float y, float x) {
  const float mx = fmaxf(y, x), mn = fminf(y, x);
  const float r = __fdividef(mn, mx), u = r * r;
  float p = 2.456720686e-03f;
  p = fmaf(p, u, -1.440134645e-02f);
  p = fmaf(p, u, 3.978121281e-02f);
  p = fmaf(p, u, -7.234857976e-02f);
  p = fmaf(p, u, 1.049894691e-01f);
  p = fmaf(p, u, -1.416122913e-01f);
  p = fmaf(p, u, 1.998590678e-01f);
  p = fmaf(p, u, -3.333259821e-01f);
  p = fmaf(p, u, 9.999998808e-01f);
  const float a = r * p;
  return y > x ? 1.57079632679f - a : a;
}

// SE3 log -> (v, w)   (se3_log, _torch_native_backend.py:289-310).  The rotation part as
// so3_log; the V^-1 coefficient c = 1/th^2 - cot(th/2) / (2 th) takes cot(th/2) = |q_w| / s
// from the quaternion itself (th / 2 = a = atan2(s, |q_w|)), so no trigonometric call is
// needed beyond the arctangent (the series of vinv_coeff below th = 1, where the closed form
// cancels).  One reciprocal r = 1/(s a) gives both th / s = 2 a^2 r and
// c = 1/(4 a^2) - |q_w| / (4 s a) = r (s^2 r - |q_w|) / 4; s and r come from the hardware
// estimates (rsqrt, reciprocal: a few ulp, far below the map's float32 conditioning).
__device__ __forceinline__ void se3_log(const Pose& T, float3& v, float3& w) {
  float4 q = T.q;
  if (q.w < 0.f) q = make_float4(-q.x, -q.y, -q.z, -q.w);
  const float s2 = q.x * q.x + q.y * q.y + q.z * q.z;
  const float qw = fminf(fmaxf(q.w, -1.f), 1.f);
  float factor, c;
  if (s2 < 0.25e-8f) {
    factor = 2.f + s2 * (2.f / 3.f);
    c = vinv_series(factor * factor * s2);
  } else {
    const float s = s2 * rsqrtf(s2);
    const float a = atan_q1(s, qw);
    const float r = __fdividef(1.f, s * a);
    factor = 2.f * (a * a) * r;
    const float th2 = 4.f * (a * a);
    c = th2 < 1.f ? vinv_series(th2) : 0.25f * r * fmaf(s2, r, -qw);
  }
  w = f3(factor * q.x, factor * q.y, factor * q.z);
  // V^-1 t = t - 1/2 w x t + c w x (w x t)
  const float3 wt = cross(w, T.t);
  v = axpy(c, cross(w, wt), axpy(-0.5f, wt, T.t));
}

// so3_exp (_torch_native_backend.py:144-159)
__device__ __forceinline__ float4 so3_exp(float3 w) {
  const float th2 = dot(w, w);
  float k, cw;
  if (th2 < 1e-8f) {
    k = 0.5f - th2 / 48.f;
    cw = 1.f - th2 / 8.f;
  } else {
    const float th = sqrtf(th2);
    float sh;
    sincosf(0.5f * th, &sh, &cw);
    k = sh / th;
  }
  return make_float4(k * w.x, k * w.y, k * w.z, cw);
}

// se3_exp for an LM increment: the same map, evaluated without trigonometric calls for
// |w| < 1 rad (Taylor series of b, c above and of sin(th/2)/th, cos(th/2), truncated where
// the next term is below float32 rounding) and with sincospif beyond.
__device__ __forceinline__ Pose se3_exp_step(float3 v, float3 w) {
  const float th2 = dot(w, w);
  float b, c, k, cw;
  if (th2 < 1.f) {
    b = fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 3628800.f, -1.f / 40320.f), 1.f / 720.f), -1.f / 24.f), 0.5f);
    c = fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 39916800.f, -1.f / 362880.f), 1.f / 5040.f), -1.f / 120.f),
             1.f / 6.f);
    const float x2 = 0.25f * th2;  // (th / 2)^2
    // sin(x)/x = 1 - x^2/6 + x^4/120 - x^6/5040 + x^8/362880; k = sin(th/2)/th = (sin(x)/x) / 2
    k = 0.5f * fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, 1.f / 362880.f, -1.f / 5040.f), 1.f / 120.f), -1.f / 6.f), 1.f);
    // cos(x) = 1 - x^2/2 + x^4/24 - x^6/720 + x^8/40320 - x^10/3628800
    cw = fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, fmaf(x2, -1.f / 3628800.f, 1.f / 40320.f), -1.f / 720.f), 1.f / 24.f),
                   -0.5f), 1.f);
  } else {
    const float th = sqrtf(th2);
    float s, co, sh;
    sincospif(th * (1.f / 3.14159265358979f), &s, &co);
    sincospif(th * (0.5f / 3.14159265358979f), &sh, &cw);
    b = 2.f * sh * sh / th2;
    c = (th - s) / (th * th2);
    k = sh / th;
  }
  const float3 wv = cross(w, v);
  Pose T;
  T.t = axpy(c, cross(w, wv), axpy(b, wv, v));
  T.q = make_float4(k * w.x, k * w.y, k * w.z, cw);
  return T;
}

// se3_exp (_torch_native_backend.py:258-286): T = (V(w) v, exp(w)).  One sincos of th/2 gives
// every coefficient (sin th = 2 sin(th/2) cos(th/2), 1 - cos th = 2 sin^2(th/2)); only
// c = (th - sin th)/th^3 cancels in float32 at small angles, so below th = 1 it comes from its
// series instead.  Selects, not branches: a warp of mixed angles runs one path.  At th = 0
// (below 1e-8 rad) the limits b = 1/2, sin(th/2)/th = 1/2, cos(th/2) = 1 are taken.
__device__ __forceinline__ Pose se3_exp(float3 v, float3 w) {
  const float th2 = dot(w, w);
  const bool tiny = th2 < 1e-16f;
  const float x = tiny ? 1.f : th2;
  const float it = rsqrtf(x), th = x * it;                 // 1 / th, th from the hardware estimate
  float sh, ch;
  sincospif(th * (0.5f / 3.14159265358979f), &sh, &ch);
  const float b = tiny ? 0.5f : 2.f * sh * sh * (it * it);
  const float k = tiny ? 0.5f : sh * it;
  const float cw = tiny ? 1.f : ch;
  const float c = th2 < 1.f ? fmaf(th2, fmaf(th2, fmaf(th2, fmaf(th2, 1.f / 39916800.f, -1.f / 362880.f),
                                                        1.f / 5040.f), -1.f / 120.f), 1.f / 6.f)
                            : (th - 2.f * sh * ch) * (it * it * it);
  const float3 wv = cross(w, v);
  Pose T;
  T.t = axpy(c, cross(w, wv), axpy(b, wv, v));
  T.q = make_float4(k * w.x, k * w.y, k * w.z, cw);
  return T;
}

// ---------------------------------------------------------------------------
// Inverse of the SE3 right Jacobian.
//
// Jr(xi) = sum_{k=0}^{N} (-1)^k/(k+1)! ad(xi)^k with ad = [[W, V], [0, W]]
// (W = hat(w), V = hat(v); tangents._ad_matrix:164-178).  The series has the
// block form [[A, B], [0, A]] with A a polynomial in W, so
// Jr^-1 = [[A^-1, -A^-1 B A^-1], [0, A^-1]].  A is kept as (a0, a1, a2) in the
// basis {I, W, W^2} (W^3 = -theta^2 W) and A^-1 as (b0, b1, b2) in the same
// basis; B is an explicit 3x3 matrix.  N = 9 reproduces the reference's
// truncated series (tangents.right_jacobian_se3:184-201, inverted with
// torch.linalg.inv at :204-207); a larger N gives the exact Jacobian.
// ---------------------------------------------------------------------------
struct JrInv {
  float3 w;          // rotation part of xi
  float b0, b1, b2;  // A^-1 = b0 I + b1 W + b2 W^2
  float B[9];        // row-major
};

// y = (b0 I + b1 W + b2 W^2) x
__device__ __forceinline__ float3 apply_poly(const float3& w, float b0, float b1, float b2, float3 x) {
  const float3 wx = cross(w, x);
  return axpy(b2, cross(w, wx), axpy(b1, wx, scale(x, b0)));
}

__device__ __forceinline__ float3 mat3_vec(const float* M, float3 x) {
  return f3(fmaf(M[0], x.x, fmaf(M[1], x.y, M[2] * x.z)), fmaf(M[3], x.x, fmaf(M[4], x.y, M[5] * x.z)),
            fmaf(M[6], x.x, fmaf(M[7], x.y, M[8] * x.z)));
}
__device__ __forceinline__ float3 mat3T_vec(const float* M, float3 x) {
  return f3(fmaf(M[0], x.x, fmaf(M[3], x.y, M[6] * x.z)), fmaf(M[1], x.x, fmaf(M[4], x.y, M[7] * x.z)),
            fmaf(M[2], x.x, fmaf(M[5], x.y, M[8] * x.z)));
}

template <int N>
__device__ __forceinline__ JrInv jr_inv_se3(float3 v, float3 w) {
  // c_k = (-1)^k / (k+1)!
  float ck[N + 1];
  {
    float f = 1.f;
#pragma unroll
    for (int k = 0; k <= N; ++k) {
      f /= (float)(k + 1);
      ck[k] = (k & 1) ? -f : f;
    }
  }
  const float th2 = dot(w, w);
  float a0 = ck[N], a1 = 0.f, a2 = 0.f;
  float B[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    // B <- W B + V A, with A = a0 I + a1 W + a2 W^2 (the previous A)
    float nB[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float3 bc = f3(B[c], B[3 + c], B[6 + c]);
      const float3 e = f3(c == 0 ? 1.f : 0.f, c == 1 ? 1.f : 0.f, c == 2 ? 1.f : 0.f);
      const float3 ac = apply_poly(w, a0, a1, a2, e);     // column c of A
      const float3 r = add(cross(w, bc), cross(v, ac));   // W B_c + V A_c
      nB[c] = r.x;
      nB[3 + c] = r.y;
      nB[6 + c] = r.z;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) B[i] = nB[i];
    // A <- c_k I + W A = c_k I + (a0 - th2 a2) W + a1 W^2
    const float na1 = fmaf(-th2, a2, a0);
    a2 = a1;
    a1 = na1;
    a0 = ck[k];
  }
  // A^-1 in the same basis: b0 = 1/a0; [m, -th2 a1; a1, m] [b1; b2] = -b0 [a1; a2], m = a0 - th2 a2
  JrInv J;
  J.w = w;
  const float b0 = 1.f / a0;
  const float m = fmaf(-th2, a2, a0);
  const float r0 = -a1 * b0, r1 = -a2 * b0;
  const float det = fmaf(m, m, th2 * a1 * a1);
  const float idet = 1.f / det;
  J.b0 = b0;
  J.b1 = (r0 * m + th2 * a1 * r1) * idet;
  J.b2 = (m * r1 - a1 * r0) * idet;
#pragma unroll
  for (int i = 0; i < 9; ++i) J.B[i] = B[i];
  return J;
}

// One column of jr_inv_se3<N>: column c of B (returned) and A^-1's coefficients b0, b1, b2.
// The columns of the series are independent given the scalar recursion of A, so three lanes can
// share one target's series; each column's arithmetic is jr_inv_se3's, in the same order.
template <int N>
__device__ __forceinline__ float3 jr_inv_se3_col(float3 v, float3 w, int c, float& b0, float& b1, float& b2) {
  float ck[N + 1];
  {
    float f = 1.f;
#pragma unroll
    for (int k = 0; k <= N; ++k) {
      f /= (float)(k + 1);
      ck[k] = (k & 1) ? -f : f;
    }
  }
  const float th2 = dot(w, w);
  float a0 = ck[N], a1 = 0.f, a2 = 0.f;
  float3 bc = f3(0.f, 0.f, 0.f);
  const float3 e = f3(c == 0 ? 1.f : 0.f, c == 1 ? 1.f : 0.f, c == 2 ? 1.f : 0.f);
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    const float3 ac = apply_poly(w, a0, a1, a2, e);     // column c of A
    bc = add(cross(w, bc), cross(v, ac));               // W B_c + V A_c
    const float na1 = fmaf(-th2, a2, a0);
    a2 = a1;
    a1 = na1;
    a0 = ck[k];
  }
  b0 = 1.f / a0;
  const float m = fmaf(-th2, a2, a0);
  const float r0 = -a1 * b0, r1 = -a2 * b0;
  const float det = fmaf(m, m, th2 * a1 * a1);
  const float idet = 1.f / det;
  b1 = (r0 * m + th2 * a1 * r1) * idet;
  b2 = (m * r1 - a1 * r0) * idet;
  return bc;
}

// out = Jr^-1 [x_lin; x_ang] = [A^-1 (x_lin - B A^-1 x_ang); A^-1 x_ang]
__device__ __forceinline__ void jr_inv_apply(const JrInv& J, float3 xl, float3 xa, float3& ol, float3& oa) {
  oa = apply_poly(J.w, J.b0, J.b1, J.b2, xa);
  ol = apply_poly(J.w, J.b0, J.b1, J.b2, sub(xl, mat3_vec(J.B, oa)));
}

// out = Jr^-T [x_lin; x_ang] = [A^-T x_lin; A^-T (x_ang - B^T A^-T x_lin)]   (A^-T: W -> -W)
__device__ __forceinline__ void jr_inv_T_apply(const JrInv& J, float3 xl, float3 xa, float3& ol, float3& oa) {
  ol = apply_poly(J.w, J.b0, -J.b1, J.b2, xl);
  oa = apply_poly(J.w, J.b0, -J.b1, J.b2, sub(xa, mat3T_vec(J.B, ol)));
}

}  // namespace br

// ---------------------------------------------------------------------------
// float64 versions for the LM accept/reject path: the iterate, forward kinematics,
// residual and cost are evaluated in double so that `cost_new < cost` is decided
// as the float64 reference decides it (levenberg_marquardt.py:114).  Same formulas
// and Taylor cutoffs as _torch_native_backend.py.
// ---------------------------------------------------------------------------
namespace br {

struct DPose {
  double3 t;
  double4 q;
};

__device__ __forceinline__ double3 d3(double x, double y, double z) { return make_double3(x, y, z); }
__device__ __forceinline__ double3 dadd(double3 a, double3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 dsub(double3 a, double3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 dscale(double3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double ddot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 dcross(double3 a, double3 b) {
  return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double4 dqmul(double4 a, double4 b) {
  double4 r;
  r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  r.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
  r.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
  r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  return r;
}
__device__ __forceinline__ double4 dqconj(double4 q) { return make_double4(-q.x, -q.y, -q.z, q.w); }
__device__ __forceinline__ double3 dqrot(double4 q, double3 p) {
  const double3 u = d3(q.x, q.y, q.z);
  const double3 c1 = dadd(dcross(u, p), dscale(p, q.w));
  return dadd(p, dscale(dcross(u, c1), 2.0));
}
__device__ __forceinline__ DPose dcompose(const DPose& a, const DPose& b) {
  DPose c;
  c.t = dadd(a.t, dqrot(a.q, b.t));
  c.q = dqmul(a.q, b.q);
  return c;
}
__device__ __forceinline__ DPose dinverse(const DPose& a) {
  DPose r;
  r.q = dqconj(a.q);
  r.t = dscale(dqrot(r.q, a.t), -1.0);
  return r;
}
__device__ __forceinline__ double4 dqnormalize(double4 q) {
  const double n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
  const double r = n2 > 1e-16 ? rsqrt(n2) : 1e8;  // 1 / max(|q|, 1e-8)
  return make_double4(q.x * r, q.y * r, q.z * r, q.w * r);
}
__device__ __forceinline__ double3 dso3_log(double4 q) {
  if (q.w < 0.0) q = make_double4(-q.x, -q.y, -q.z, -q.w);
  const double s2 = q.x * q.x + q.y * q.y + q.z * q.z;
  const double s = sqrt(s2);
  double factor;
  if (s2 < 1e-8 / 4.0) {
    factor = 2.0 + s2 * (2.0 / 3.0);
  } else {
    factor = 2.0 * atan2(s, fmin(fmax(q.w, -1.0), 1.0)) / s;
  }
  return d3(factor * q.x, factor * q.y, factor * q.z);
}
__device__ __forceinline__ void dse3_log(const DPose& T, double3& v, double3& w) {
  // the rotation part as dso3_log: w = f q_xyz with f = 2 atan2(s, |q_w|) / s, s = |q_xyz|
  double4 q = T.q;
  if (q.w < 0.0) q = make_double4(-q.x, -q.y, -q.z, -q.w);
  const double s2 = q.x * q.x + q.y * q.y + q.z * q.z;
  // c = 1/th^2 - cot(th/2) / (2 th) with th = 2a, a = atan2(s, |q_w|), s = |q_xyz|, and
  // cot(th/2) = |q_w| / s exactly (no trigonometric call): c = (1 - a |q_w| / s) / (4 a^2);
  // f = 2a / s.  One division: r = 1 / (a s) gives 1/s = a r and 1/a = s r.
  double f, c = 0.0;
  const bool small = s2 < 1e-8 / 4.0;
  if (small) {
    f = 2.0 + s2 * (2.0 / 3.0);
  } else {
    const double s = sqrt(s2);
    const double a = atan2(s, fmin(q.w, 1.0));
    const double r = 1.0 / (a * s);
    const double ar = a * a * r;  // a / s
    const double sr = s * r;      // 1 / a
    f = 2.0 * ar;
    c = fma(-ar, q.w, 1.0) * (0.25 * sr * sr);
  }
  w = d3(f * q.x, f * q.y, f * q.z);
  const double th2 = ddot(w, w);
  if (small || th2 < 1e-8) c = 1.0 / 12.0 + th2 / 720.0;
  const double3 wt = dcross(w, T.t);
  v = dadd(dadd(T.t, dscale(wt, -0.5)), dscale(dcross(w, wt), c));
}
__device__ __forceinline__ DPose dse3_exp(double3 v, double3 w) {
  const double th2 = ddot(w, w);
  double b, c, k, cw;
  if (th2 < 1e-8) {
    b = 0.5 - th2 / 24.0;
    c = 1.0 / 6.0 - th2 / 120.0;
    k = 0.5 - th2 / 48.0;
    cw = cos(0.5 * sqrt(th2));
  } else {
    const double th = sqrt(th2);
    double s, co, sh;
    sincos(th, &s, &co);
    sincos(0.5 * th, &sh, &cw);
    b = (1.0 - co) / th2;
    c = (th - s) / (th * th2);
    k = sh / th;
  }
  const double3 wv = dcross(w, v);
  DPose T;
  T.t = dadd(dadd(v, dscale(wv, b)), dscale(dcross(w, wv), c));
  T.q = make_double4(k * w.x, k * w.y, k * w.z, cw);
  return T;
}

}  // namespace br

// float64 SE3 Jr^-1 (same block-Horner construction as jr_inv_se3 above), used where the
// normal equations are ill-conditioned enough that float32 Jacobian rounding is amplified
// (the trajectory problem, condition ~1e8).
namespace br {

struct DJrInv {
  double3 w;
  double b0, b1, b2;
  double B[9];
};

__device__ __forceinline__ double3 dapply_poly(const double3& w, double b0, double b1, double b2, double3 x) {
  const double3 wx = dcross(w, x);
  return dadd(dadd(dscale(x, b0), dscale(wx, b1)), dscale(dcross(w, wx), b2));
}

template <int N>
__device__ __forceinline__ DJrInv djr_inv_se3(double3 v, double3 w) {
  double ck[N + 1];
  {
    double f = 1.0;
#pragma unroll
    for (int k = 0; k <= N; ++k) {
      f /= (double)(k + 1);
      ck[k] = (k & 1) ? -f : f;
    }
  }
  const double th2 = ddot(w, w);
  double a0 = ck[N], a1 = 0.0, a2 = 0.0;
  double B[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    double nB[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double3 bc = d3(B[c], B[3 + c], B[6 + c]);
      const double3 e = d3(c == 0 ? 1.0 : 0.0, c == 1 ? 1.0 : 0.0, c == 2 ? 1.0 : 0.0);
      const double3 ac = dapply_poly(w, a0, a1, a2, e);
      const double3 r = dadd(dcross(w, bc), dcross(v, ac));
      nB[c] = r.x; nB[3 + c] = r.y; nB[6 + c] = r.z;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) B[i] = nB[i];
    const double na1 = a0 - th2 * a2;
    a2 = a1;
    a1 = na1;
    a0 = ck[k];
  }
  DJrInv J;
  J.w = w;
  const double b0 = 1.0 / a0;
  const double m = a0 - th2 * a2;
  const double r0 = -a1 * b0, r1 = -a2 * b0;
  const double idet = 1.0 / (m * m + th2 * a1 * a1);
  J.b0 = b0;
  J.b1 = (r0 * m + th2 * a1 * r1) * idet;
  J.b2 = (m * r1 - a1 * r0) * idet;
#pragma unroll
  for (int i = 0; i < 9; ++i) J.B[i] = B[i];
  return J;
}

// One column of djr_inv_se3<N> (see jr_inv_se3_col).
template <int N>
__device__ __forceinline__ double3 djr_inv_se3_col(double3 v, double3 w, int c, double& b0, double& b1, double& b2) {
  double ck[N + 1];
  {
    double f = 1.0;
#pragma unroll
    for (int k = 0; k <= N; ++k) {
      f /= (double)(k + 1);
      ck[k] = (k & 1) ? -f : f;
    }
  }
  const double th2 = ddot(w, w);
  double a0 = ck[N], a1 = 0.0, a2 = 0.0;
  double3 bc = d3(0.0, 0.0, 0.0);
  const double3 e = d3(c == 0 ? 1.0 : 0.0, c == 1 ? 1.0 : 0.0, c == 2 ? 1.0 : 0.0);
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    const double3 ac = dapply_poly(w, a0, a1, a2, e);
    bc = dadd(dcross(w, bc), dcross(v, ac));
    const double na1 = a0 - th2 * a2;
    a2 = a1;
    a1 = na1;
    a0 = ck[k];
  }
  b0 = 1.0 / a0;
  const double m = a0 - th2 * a2;
  const double r0 = -a1 * b0, r1 = -a2 * b0;
  const double idet = 1.0 / (m * m + th2 * a1 * a1);
  b1 = (r0 * m + th2 * a1 * r1) * idet;
  b2 = (m * r1 - a1 * r0) * idet;
  return bc;
}

__device__ __forceinline__ void djr_inv_apply(const DJrInv& J, double3 xl, double3 xa, double3& ol, double3& oa) {
  oa = dapply_poly(J.w, J.b0, J.b1, J.b2, xa);
  const double3 Bo = d3(J.B[0] * oa.x + J.B[1] * oa.y + J.B[2] * oa.z, J.B[3] * oa.x + J.B[4] * oa.y + J.B[5] * oa.z,
                        J.B[6] * oa.x + J.B[7] * oa.y + J.B[8] * oa.z);
  ol = dapply_poly(J.w, J.b0, J.b1, J.b2, dsub(xl, Bo));
}

__device__ __forceinline__ void djr_inv_T_apply(const DJrInv& J, double3 xl, double3 xa, double3& ol, double3& oa) {
  ol = dapply_poly(J.w, J.b0, -J.b1, J.b2, xl);
  const double3 Bt = d3(J.B[0] * ol.x + J.B[3] * ol.y + J.B[6] * ol.z, J.B[1] * ol.x + J.B[4] * ol.y + J.B[7] * ol.z,
                        J.B[2] * ol.x + J.B[5] * ol.y + J.B[8] * ol.z);
  oa = dapply_poly(J.w, J.b0, -J.b1, J.b2, dsub(xa, Bt));
}

}  // namespace br

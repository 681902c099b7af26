// SPDX-License-Identifier: Apache-2.0
// Scalar SPH math on the device: kernel value and gradient factor, half-space boundary volume, colour inversion.
//
// Arithmetic contract: every expression below has a fixed evaluation order, explicit fused multiply-adds
// (__fmaf_rn) and IEEE sqrt and division; the library is compiled with -fmad=false so that nothing else is fused.
// The CPU oracle evaluates the same expressions in the same order, so the two agree bit for bit.
#pragma once

#include <cuda_runtime.h>

namespace adf {

#define ADF_FMA(a, b, c) __fmaf_rn((a), (b), (c))

// Packed pairs of floats for sm_100's two-wide FP32 instructions (add/sub/mul.rn.f32x2): each half is rounded as the
// scalar instruction would round it. The assembler may still contract a packed multiply whose only use is a packed
// add into a fused multiply-add (observed on sm_100a even with -fmad=false), so bit-exact code uses the packed
// subtraction and keeps products and their sums scalar.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_dup(float a) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ f32x2 f2_load(const float* p) {  // p 8-byte aligned: p[0] low half, p[1] high half
  return *reinterpret_cast<const f32x2*>(p);
}
__device__ __forceinline__ float f2_lo(f32x2 a) {
  float lo;
  asm("{\n\t.reg .b32 hi;\n\tmov.b64 {%0, hi}, %1;\n\t}" : "=f"(lo) : "l"(a));
  return lo;
}
__device__ __forceinline__ float f2_hi(f32x2 a) {
  float hi;
  asm("{\n\t.reg .b32 lo;\n\tmov.b64 {lo, %0}, %1;\n\t}" : "=f"(hi) : "l"(a));
  return hi;
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

struct KC {
  int kind;  // 0 cubic spline, 1 Wendland C2
  float h, inv_h, h2, sigma, sig_h2, m6sig_h, m20sig_h2, r_min;
};

inline KC make_kc(int kind, double h, double sigma) {
  KC k;
  k.kind = kind;
  k.h = (float)h;
  k.inv_h = (float)(1.0 / h);
  k.h2 = k.h * k.h;
  k.sigma = (float)sigma;
  k.sig_h2 = (float)(sigma / (h * h));
  k.m6sig_h = (float)(-6.0 * sigma / h);
  k.m20sig_h2 = (float)(-20.0 * sigma / (h * h));
  k.r_min = (float)(1.0e-9 * h);
  return k;
}

__device__ __forceinline__ float maxr(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minr(float a, float b) { return a < b ? a : b; }

// the reference's dot (left to right, no fusion): pair distances
__device__ __forceinline__ float dot_plain(float ax, float ay, float az, float bx, float by, float bz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}
// fused dot used everywhere else
__device__ __forceinline__ float dotf(float ax, float ay, float az, float bx, float by, float bz) {
  return ADF_FMA(az, bz, ADF_FMA(ay, by, __fmul_rn(ax, bx)));
}

// W(r) and F(r) = (dW/dr)/r from r^2 (kernels.py:41-77); grad W_ij = (x_i - x_j) F.
__device__ __forceinline__ void wf(const KC& k, float r2, float& W, float& F) {
  float r = __fsqrt_rn(r2);
  float q = __fmul_rn(r, k.inv_h);
  if (q >= 1.0f) { W = 0.0f; F = 0.0f; return; }
  if (k.kind == 0) {
    if (q <= 0.5f) {
      W = __fmul_rn(k.sigma, ADF_FMA(__fmul_rn(6.0f, __fmul_rn(q, q)), __fsub_rn(q, 1.0f), 1.0f));
      F = __fmul_rn(k.sig_h2, ADF_FMA(18.0f, q, -12.0f));
    } else {
      float s = __fsub_rn(1.0f, q);
      float s2 = __fmul_rn(s, s);
      W = __fmul_rn(k.sigma, __fmul_rn(2.0f, __fmul_rn(s2, s)));
      F = __fdiv_rn(__fmul_rn(k.m6sig_h, s2), r);
    }
  } else {
    float s = __fsub_rn(1.0f, q);
    float s2 = __fmul_rn(s, s);
    W = __fmul_rn(k.sigma, __fmul_rn(__fmul_rn(s2, s2), ADF_FMA(4.0f, q, 1.0f)));
    F = __fmul_rn(k.m20sig_h2, __fmul_rn(s2, s));
  }
  if (r <= k.r_min) F = 0.0f;
}

// Psi(d) and dPsi/dd of a flat solid half-space at signed distance d (kernels.py:80-138, curvature 0).
__device__ __forceinline__ void halfspace(const KC& k, float d, float& psi, float& dpsi) {
  if (d >= k.h) { psi = 0.0f; dpsi = 0.0f; return; }
  float z = minr(maxr(__fmul_rn(-d, k.inv_h), -1.0f), 1.0f);
  float y = fabsf(z);
  float g0, p;
  if (k.kind == 0) {
    if (y <= 0.5f) {
      float y2 = __fmul_rn(y, y);
      g0 = __fmul_rn(y, ADF_FMA(y2, ADF_FMA(y2, ADF_FMA((float)(-3.2), y, (float)(4.8)), (float)(-2.66666666666666667)),
                                (float)(1.4)));
      p = ADF_FMA(y2, ADF_FMA(y2, ADF_FMA((float)(-19.2), y, 24.0f), -8.0f), (float)(1.4));
    } else {
      float u = __fsub_rn(1.0f, y);
      float u2 = __fmul_rn(u, u);
      float u4 = __fmul_rn(u2, u2);
      g0 = __fsub_rn(0.5f, __fmul_rn(__fmul_rn(u4, u), ADF_FMA((float)(-1.06666666666666667), u, (float)(1.6))));
      p = __fmul_rn(u4, ADF_FMA((float)(6.4), y, (float)(1.6)));
    }
  } else {
    float y2 = __fmul_rn(y, y);
    g0 = __fmul_rn(y, ADF_FMA(y2, ADF_FMA(y2, ADF_FMA(y, ADF_FMA(y, ADF_FMA(-1.5f, y, 7.5f), -14.0f), 10.5f), -3.5f),
                              1.5f));
    p = ADF_FMA(y2, ADF_FMA(y2, ADF_FMA(y, ADF_FMA(y, ADF_FMA(-12.0f, y, 52.5f), -84.0f), 52.5f), -10.5f), 1.5f);
  }
  psi = (z < 0.0f) ? __fsub_rn(0.5f, g0) : __fadd_rn(0.5f, g0);
  dpsi = (d > -k.h) ? __fmul_rn(-p, k.inv_h) : 0.0f;
}

// The distance at which a flat wall covers c of the support (particle_walls.py:87-98): 30 bisection steps.
__device__ __forceinline__ float colour_distance(const KC& k, float c) {
  float lo = -k.h, hi = k.h;
#pragma unroll 1
  for (int it = 0; it < 30; ++it) {
    float mid = __fmul_rn(0.5f, __fadd_rn(lo, hi));
    float psi, dpsi;
    halfspace(k, mid, psi, dpsi);
    if (psi > c) lo = mid; else hi = mid;
  }
  return __fmul_rn(0.5f, __fadd_rn(lo, hi));
}

// q' = q rotated by the unit quaternion (qx, qy, qz, qw): v (2w^2 - 1) + 2w (u x v) + 2u (u . v)
__device__ __forceinline__ void quat_rotate(const float* qv, float vx, float vy, float vz, float& ox, float& oy,
                                            float& oz) {
  float ux = qv[0], uy = qv[1], uz = qv[2], w = qv[3];
  float a = __fsub_rn(__fmul_rn(2.0f, __fmul_rn(w, w)), 1.0f);
  float cx = __fsub_rn(__fmul_rn(uy, vz), __fmul_rn(uz, vy));
  float cy = __fsub_rn(__fmul_rn(uz, vx), __fmul_rn(ux, vz));
  float cz = __fsub_rn(__fmul_rn(ux, vy), __fmul_rn(uy, vx));
  float b = __fmul_rn(2.0f, w);
  float d = __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(ux, vx), __fmul_rn(uy, vy)), __fmul_rn(uz, vz)));
  ox = __fadd_rn(__fadd_rn(__fmul_rn(vx, a), __fmul_rn(cx, b)), __fmul_rn(ux, d));
  oy = __fadd_rn(__fadd_rn(__fmul_rn(vy, a), __fmul_rn(cy, b)), __fmul_rn(uy, d));
  oz = __fadd_rn(__fadd_rn(__fmul_rn(vz, a), __fmul_rn(cz, b)), __fmul_rn(uz, d));
}

__device__ __forceinline__ long long to_fixed(float m) { return llround((double)m * 1099511627776.0); }

}  // namespace adf

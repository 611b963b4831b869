// Device arithmetic of the formal solvers and the line opacity, sm_100a.
//
// The library is compiled with -fmad=false: every fused multiply-add below is
// an explicit fmaf()/fma(), so the FP32 results are one fixed evaluation of the
// reference's real(4) expressions and agree bit for bit with any other
// evaluation that makes the same choices.
//
//   exp_neg / exp_neg0 / exp4      HOP/exp_neg.inc:20-74
//   lw_series / linear_weights     SRC/rt_solvers_mod.f90:785-845
//   parab_moments                  SRC/rt_solvers_mod.f90:862-877
//
// The FP64 twins (T = double) use exact exp/expm1 with Taylor forms where the
// closed forms cancel; they are the plain FP64 path.
#pragma once
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace m3d {

// exp(-t), 1 - exp(-t); t clamped at 87 (exp_neg.inc:20-39)
__device__ __forceinline__ void exp_neg(float t, float &E, float &u0) {
  const float tc = fminf(t, 87.0f);
  const float n = roundf(tc * 1.44269504f);
  const float r = fmaf(-n, -2.12194440e-4f, fmaf(-n, 0.693359375f, tc));
  float p = fmaf(r, -1.351550105e-03f, +8.353385143e-03f);
  p = fmaf(r, p, -4.167019576e-02f);
  p = fmaf(r, p, +1.666666716e-01f);
  p = fmaf(r, p, -5.000000000e-01f);
  p = fmaf(r, p, +1.000000000e+00f);
  const float m = r * p;
  const float s = __uint_as_float((uint32_t)(127 - (int)n) << 23);
  E = s * (1.0f - m);
  u0 = fmaf(s, m, 1.0f - s);
}

// exp_neg0: E = 0 above t = 87 (and for a NaN t), t clamped at -87 below (exp_neg.inc:41-51)
__device__ __forceinline__ void exp_neg0(float t, float &E, float &u0) {
  exp_neg(fmaxf(t, -87.0f), E, u0);
  if (!(t <= 87.0f)) E = 0.0f;
}

// exp4(x) = exp_neg0(-x): 0 below x = -87, saturating at exp(87) (exp_neg.inc:45-62)
__device__ __forceinline__ float exp4(float x) {
  const float t = -x;
  float E, u0;
  exp_neg(fmaxf(t, -87.0f), E, u0);
  return (t <= 87.0f) ? E : 0.0f;
}

// fp32 log from the atanh series: x = 2^e m, m in [sqrt(1/2), sqrt(2)),
// log m = 2 atanh(s), s = (m-1)/(m+1), series to s^11; e ln2 with a split ln2.
__device__ __forceinline__ float logf_m3d(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : __int_as_float(0x7fc00000);
  if (x == INFINITY) return x;
  int e = 0;
  if (x < FLT_MIN) { x = x * 8388608.0f; e = -23; }
  const uint32_t u = __float_as_uint(x);
  e += (int)((u >> 23) & 0xff) - 127;
  float m = __uint_as_float((u & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
  const float f = m - 1.0f;
  const float s = f / (2.0f + f);
  const float s2 = s * s;
  float p = fmaf(s2, 0.0909090936f, 0.111111112f);
  p = fmaf(s2, p, 0.142857143f);
  p = fmaf(s2, p, 0.200000003f);
  p = fmaf(s2, p, 0.333333343f);
  p = fmaf(s2, p, 1.0f);
  const float lm = (2.0f * s) * p;
  const float fe = (float)e;
  const float r = fmaf(fe, 1.42860677e-06f, lm);
  return fmaf(fe, 0.693145752f, r);
}

__device__ __forceinline__ float lw_series(float t) {
  float p = fmaf(t, -2.834696488e-06f, +2.522676368e-05f);
  p = fmaf(t, p, -1.983609400e-04f);
  p = fmaf(t, p, +1.388740959e-03f);
  p = fmaf(t, p, -8.333330974e-03f);
  p = fmaf(t, p, +4.166666791e-02f);
  p = fmaf(t, p, -1.666666716e-01f);
  p = fmaf(t, p, +5.000000000e-01f);
  return t * p;
}

// E, W, Psi, Esc of the linear step over optical depth t
__device__ __forceinline__ void linear_weights(float t, float &E, float &W, float &Psi, float &Esc) {
  float u0;
  exp_neg(t, E, u0);
  const float ut = u0 / t;
  const float ps = lw_series(t);
  const bool thin = fabsf(t) <= 1.0f;
  Psi = thin ? ps : 1.0f - ut;
  Esc = thin ? 1.0f - ps : ut;
  W = thin ? u0 - ps : ut - E;
}

// bezier3_weights (rt_solvers_mod.f90:1280-1304): the cubic-Bezier weights over
// optical depth t, w_k = t int_0^1 b_k(u) exp(-t u) du, b = u^3, 3u^2(1-u),
// 3u(1-u)^2, (1-u)^3.  For t <= 3 the series t E P3(-t), t E P2(-t), t P2(t),
// t P3(t), P2 and P3 the reference's minimax fits (b3_p2, b3_p3, :1305-1331);
// above, the moments M_n = n M_(n-1) - t^n E from M0 = 1 - E at max(t, 3).
__device__ __forceinline__ float b3_p2(float t) {
  float p = fmaf(t, +7.658396139e-10f, -1.100420821e-08f);
  p = fmaf(t, p, +1.137804801e-07f);
  p = fmaf(t, p, -1.190877015e-06f);
  p = fmaf(t, p, +1.156294547e-05f);
  p = fmaf(t, p, -9.924791084e-05f);
  p = fmaf(t, p, +7.440865738e-04f);
  p = fmaf(t, p, -4.761847202e-03f);
  p = fmaf(t, p, +2.499995567e-02f);
  p = fmaf(t, p, -1.000000238e-01f);
  return fmaf(t, p, +2.500000000e-01f);
}
__device__ __forceinline__ float b3_p3(float t) {
  float p = fmaf(t, -1.025371787e-09f, +1.414234507e-08f);
  p = fmaf(t, p, -1.503805294e-07f);
  p = fmaf(t, p, +1.640762775e-06f);
  p = fmaf(t, p, -1.653099389e-05f);
  p = fmaf(t, p, +1.488493726e-04f);
  p = fmaf(t, p, -1.190488110e-03f);
  p = fmaf(t, p, +8.333289996e-03f);
  p = fmaf(t, p, -4.999998957e-02f);
  return fmaf(t, p, +2.500000000e-01f);
}
__device__ __forceinline__ void bezier3_weights(float t, float &E, float &w0, float &w1, float &w2, float &w3) {
  const float tser = 3.0f;
  float M0;
  exp_neg(t, E, M0);
  const float tb = fmaxf(t, tser);
  const float tb2 = tb * tb;
  const float tb3 = tb2 * tb;
  const float r3 = 1.0f / tb3;
  const float M1 = fmaf(-tb, E, M0);
  const float M2 = fmaf(-tb2, E, 2.0f * M1);
  const float M3 = fmaf(-tb3, E, 3.0f * M2);
  const float b0 = M3 * r3;
  const float b1 = (3.0f * fmaf(M2, tb, -M3)) * r3;
  const float b2 = (3.0f * (fmaf(M1, tb2, -((2.0f * M2) * tb)) + M3)) * r3;
  const bool ser = t <= tser;
  const float tE = t * E;
  w0 = ser ? tE * b3_p3(-t) : b0;
  w1 = ser ? tE * b3_p2(-t) : b1;
  w2 = ser ? t * b3_p2(t) : b2;
  w3 = ser ? t * b3_p3(t) : ((M0 - b0) - b1) - b2;
}

// Taylor sums of the FP64 forms below |t| = 0.1 where the closed forms cancel:
// sum_{k=k0}^{k0+11} scale (-1)^k t^(k-shift)/k!  (Psi: k0=2, shift=1; U1: k0=2,
// shift=0; q: k0=3, shift=1, scale=-2), truncation below 1e-17 relative.
__device__ __forceinline__ double series64(double t, int k0, int shift, double scale) {
  double fact = 1.0;
  for (int k = 2; k <= k0 + 11; k++) fact *= k;
  double p = 0.0;
  for (int k = k0 + 11; k >= k0; k--) {
    p = p * t + ((k & 1) ? -1.0 : 1.0) / fact;
    fact /= (k > 1 ? k : 1);
  }
  double tp = 1.0;
  for (int k = 0; k < k0 - shift; k++) tp *= t;
  return scale * p * tp;
}

__device__ __forceinline__ void linear_weights(double t, double &E, double &W, double &Psi, double &Esc) {
  const double tc = fmin(t, 700.0);
  E = exp(-tc);
  const double u0 = -expm1(-tc);
  if (fabs(t) < 0.1) {
    const double ps = series64(t, 2, 1, 1.0);
    Psi = ps;
    Esc = 1.0 - ps;
    W = u0 - ps;
  } else {
    const double ut = u0 / t;
    Psi = 1.0 - ut;
    Esc = ut;
    W = ut - E;
  }
}

// E, U0 = 1-E, U1 = t-U0, q = (t^2 - 2 U1)/t
__device__ __forceinline__ void parab_moments(float t, float &E, float &U0, float &U1, float &q) {
  exp_neg(t, E, U0);
  U1 = fabsf(t) <= 1.0f ? t * lw_series(t) : t - U0;
  float p = fmaf(t, +5.153443894e-08f, -5.894584660e-07f);
  p = fmaf(t, p, +5.514686109e-06f);
  p = fmaf(t, p, -4.948913192e-05f);
  p = fmaf(t, p, +3.968053206e-04f);
  p = fmaf(t, p, -2.777901944e-03f);
  p = fmaf(t, p, +1.666668802e-02f);
  p = fmaf(t, p, -8.333329856e-02f);
  p = fmaf(t, p, +3.333333433e-01f);
  const float qs = (t * t) * p;
  q = fabsf(t) <= 2.0f ? qs : t - 2.0f * (U1 / t);
}

__device__ __forceinline__ void parab_moments(double t, double &E, double &U0, double &U1, double &q) {
  const double tc = fmin(t, 700.0);
  E = exp(-tc);
  U0 = -expm1(-tc);
  if (fabs(t) < 0.1) {
    U1 = series64(t, 2, 0, 1.0);
    q = series64(t, 3, 1, -2.0);
  } else {
    U1 = t - U0;
    q = t - 2.0 * (U1 / t);
  }
}

// ---- packed FP32 pairs (sm_100's f32x2 add/mul/fma) ------------------------
// Each half is rounded exactly as the scalar instruction rounds it (IEEE, round to
// nearest even unless the name says otherwise), so a pair evaluation is bit-identical
// to two scalar ones; it takes one issue slot instead of two.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void up2(f32x2 v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// a + b rounded toward zero
__device__ __forceinline__ f32x2 add2_rz(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ f32x2 splat2(float v) { return pk2(v, v); }

template <typename T> __device__ __forceinline__ T tiny_of();
template <> __device__ __forceinline__ float tiny_of<float>() { return FLT_MIN; }
template <> __device__ __forceinline__ double tiny_of<double>() { return DBL_MIN; }

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }

}  // namespace m3d

// QLG-bot Voigt profile on the device (HOP/qlg_mod.f90, OpenMULTI3D's additions
// bot_setup :538, qlg_bot_line_eval :556, qlg_bot_cell :576, qlg_bot_line :616,
// qlg_bot_line_sweep :646).  The two tables TGX = 2^-u and TH2X = Z_0.2(u)(1+u)^2
// (qlg_init :364) live in global memory and are staged into shared memory by the
// kernels that sweep line windows.  The fitted constants are the published QLG-bot
// coefficients; they have to be the same numbers for the profile to be QLG-bot.
//
// The tables are read interleaved, tab[i] = (TGX(i), TH2X(i)), one 8-byte load per
// point.  Two exact rewrites keep the point cost down: 1/(1+u) is the correctly
// rounded reciprocal (__frcp_rn equals the IEEE quotient 1.0f/(1+u)), and the
// snapped index nint(min(xs*800, 9019)) is floor(y + 0.5), taken from the bits of
// RZ(RZ(y + 0.5) + 2^23) (qlg_node) without a float-to-int conversion.
#pragma once
#include "m3d_math.cuh"

namespace m3d {

constexpr int QLG_NTAB = 9020;  // indices 0..9019 on xi = sqrt(u) at 800 per unit

struct QlgCoef { float ih, bL, gG, cZH, cL2; };
struct QlgCell { float D, D2, SQ, D2h, D2G, D2L; };

__device__ __forceinline__ QlgCell qlg_cell(float D) {
  QlgCell w;
  w.D = D;
  w.D2 = D * D;
  w.SQ = 0.8325546112f * w.D2;
  w.D2h = 0.5f * w.D2;
  w.D2G = 1.5f * w.D2;
  w.D2L = 5.0f * w.D2;
  return w;
}

// per-line setup on the caller's abscissa: gL Lorentz width, D Doppler width,
// SQ = sqrt(ln2) D^2, S the strength folded in
__device__ __forceinline__ QlgCoef qlg_setup(float gL, float D, float SQ, float S) {
  QlgCoef c;
  const float e = fmaf(gL, 0.60602209212341318f, D);
  c.ih = e / fmaf(gL, e, SQ);
  const float r = gL * c.ih;
  const float q = r * (1.0f - r);
  const float sc = S * c.ih;
  const float qs = q * sc;
  const float x = 2.0f * r - 1.0f;
  c.bL = (0.3183098862f * r) * sc;
  c.gG = fmaf(qs, fmaf(x, -0.11019326278794868f, -0.064924393191013452f), (0.4697186f * (1.0f - r)) * sc);
  c.cZH = qs * fmaf(x, -0.10567135279610407f, 0.38494195930078284f);
  c.cL2 = qs * fmaf(x, 0.16241029253712097f, 0.04054415746208978f);
  return c;
}

// 1/d correctly rounded for d in [1, 2^126): the approximate reciprocal refined by
// one Newton step in fused multiply-adds, e = 1 - d r, r + r e (Markstein's method,
// IBM J. Res. Dev. 34 (1990) 111).  Equal to __frcp_rn on every float of that range
// (an exhaustive comparison on the B200); beyond it the approximation flushes to
// zero, so callers bound d first.
__device__ __forceinline__ float rcp_markstein(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  const float e = fmaf(-d, r, 1.0f);
  return fmaf(r, e, r);
}

// the correctly rounded reciprocal of d >= 1: MK when the caller has bounded d below 2^126
template <bool MK>
__device__ __forceinline__ float qlg_rcp(float d) {
  if (MK) return rcp_markstein(d);
  return __frcp_rn(d);
}

// the snapped table node nint(y) of y = min(xs 800, 9019) >= 0 (NaN included: fminf
// returns 9019): floor(y + 0.5), which is floor(RZ(y + 0.5)) since rounding toward
// zero never carries a positive sum past the integer below it; adding 2^23 toward
// zero then leaves that integer in the low mantissa bits.  Two additions and an
// integer subtraction, no float-to-int conversion; equal to (int)(y + 0.5f) with
// y < 0.5 sent to node 0 for every y in [0, 9019].
__device__ __forceinline__ int qlg_node(float y) {
  return __float_as_int(__fadd_rz(__fadd_rz(y, 0.5f), 8388608.0f)) - 0x4B000000;
}

template <bool MK = false>
__device__ __forceinline__ float qlg_eval(const float2 *tab, const QlgCoef &c, float x) {
  const float xs = fabsf(x) * c.ih;
  const float u = xs * xs;
  const float L = qlg_rcp<MK>(1.0f + u);
  const float y = fminf(xs * 800.0f, 9019.0f);
  const float2 gw = tab[qlg_node(y)];
  const float G = gw.x, W = gw.y;
  float p = fmaf(c.cZH, W, c.cL2);
  p = fmaf(L, p, c.bL);
  return fmaf(L, p, G * c.gG);
}

// analytic half-width where the line falls to ref (qlg_bot_line, qlg_mod.f90:616-627)
__device__ __forceinline__ float qlg_halfwidth(const QlgCell &w, float gL, float S, float ref, float lnq) {
  const float AL = ((0.3183098862f * gL) * S) / ref;
  const float h1 = fmaf(w.D2, lnq, fminf(AL, w.D2G));
  const float h2 = (AL - fmaxf(fmaf(gL, gL, -w.D2h), 0.0f)) + fminf(AL, w.D2L);
  return sqrtf(fmaxf(fmaxf(h1, h2), 0.0f));
}

}  // namespace m3d

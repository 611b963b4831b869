/*
 * m3d_oracle.c -- CPU restatement of OpenMULTI3D's radiative-transfer hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the CUDA library, loaded by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.  Nothing in the
 * product links or calls it.  Build: oracle/Makefile (gcc -O2 -ffp-contract=off).
 *
 * Each routine cites the reference routine (file:line, paths relative to
 * experiments/OpenMULTI3D/) whose arithmetic it restates.  Where the reference
 * calls the platform libm exp/log on a path that decides an integer (a line's
 * window), this file uses the reference's own fp32 exponential (exp_neg.inc)
 * and an fp32 logarithm from the atanh series, written out op by op, so that
 * the CUDA kernels can reproduce window indices bit for bit.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "m3d_oracle.h"

/* const_mod.f90:38-73 */
#define OR_HH 6.626176e-27
#define OR_BK 1.380662e-16
#define OR_CC 2.99792458e10
#define OR_PI 3.14159265359
#define OR_H_K (OR_HH / OR_BK)
#define OR_CM_TO_AA 1e8

static inline float f32_from_bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t bits_from_f32(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* =========================================================================
 * K0: exp_neg, exp_neg0, exp4 (HOP/exp_neg.inc:20-74)
 * ========================================================================= */
static const float EXP_LOG2E = 1.44269504f, EXP_C1 = 0.693359375f, EXP_C2 = -2.12194440e-4f;
static const float EXP_Q[6] = {+1.000000000e+00f, -5.000000000e-01f, +1.666666716e-01f,
                               -4.167019576e-02f, +8.353385143e-03f, -1.351550105e-03f};

/* exp(-t) and 1-exp(-t), neither formed from the other; t clamped at 87 */
static inline void or_exp_neg1(float t, float *E, float *u0)
{
  float tc = fminf(t, 87.0f);
  float n = roundf(tc * EXP_LOG2E);
  float r = fmaf(-n, EXP_C2, fmaf(-n, EXP_C1, tc));
  float p = fmaf(r, EXP_Q[5], EXP_Q[4]);
  p = fmaf(r, p, EXP_Q[3]);
  p = fmaf(r, p, EXP_Q[2]);
  p = fmaf(r, p, EXP_Q[1]);
  p = fmaf(r, p, EXP_Q[0]);
  float m = r * p;
  float s = f32_from_bits((uint32_t)(127 - (int)n) << 23);
  *E = s * (1.0f - m);
  *u0 = fmaf(s, m, 1.0f - s);
}

/* exp_neg0: E = 0 above t = 87, t clamped at -87 below */
static inline void or_exp_neg0(float t, float *E, float *u0)
{
  or_exp_neg1(fmaxf(t, -87.0f), E, u0);
  if (!(t <= 87.0f)) *E = 0.0f;
}

/* exp4(x) = exp_neg0(-x) */
static inline float or_exp4(float x)
{
  float E, u0;
  or_exp_neg0(-x, &E, &u0);
  return E;
}

/* fp32 natural log for x > 0: x = 2^e m, m in [sqrt(1/2), sqrt(2)), log m =
 * 2 atanh(s), s = (m-1)/(m+1), by its Taylor series to s^11 (|s| <= 0.1716);
 * e ln2 with ln2 split so that e*LN2_HI is exact.  Used wherever the
 * reference's libm log feeds a window index (logref, the floored reference,
 * the van der Waals power). */
static inline float or_logf1(float x)
{
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int e = 0;
  if (x < FLT_MIN) { x *= 8388608.0f; e = -23; }
  uint32_t u = bits_from_f32(x);
  e += (int)((u >> 23) & 0xff) - 127;
  float m = f32_from_bits((u & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421356f) { m *= 0.5f; e += 1; }
  float f = m - 1.0f;
  float s = f / (2.0f + f);
  float s2 = s * s;
  float p = fmaf(s2, 0.0909090936f, 0.111111112f);   /* 1/11, 1/9 */
  p = fmaf(s2, p, 0.142857143f);                       /* 1/7 */
  p = fmaf(s2, p, 0.200000003f);                       /* 1/5 */
  p = fmaf(s2, p, 0.333333343f);                       /* 1/3 */
  p = fmaf(s2, p, 1.0f);
  float lm = (2.0f * s) * p;
  float fe = (float)e;
  float r = fmaf(fe, 1.42860677e-06f, lm);             /* ln2 - LN2_HI */
  return fmaf(fe, 0.693145752f, r);                    /* LN2_HI = 0x3f317200 */
}

void or_exp_neg_f32(int n, const float *t, float *E, float *u0)
{
  for (int i = 0; i < n; i++) or_exp_neg1(t[i], &E[i], &u0[i]);
}
void or_exp_neg0_f32(int n, const float *t, float *E, float *u0)
{
  for (int i = 0; i < n; i++) or_exp_neg0(t[i], &E[i], &u0[i]);
}
void or_exp4_f32(int n, const float *x, float *y)
{
  for (int i = 0; i < n; i++) y[i] = or_exp4(x[i]);
}
void or_log_f32(int n, const float *x, float *y)
{
  for (int i = 0; i < n; i++) y[i] = or_logf1(x[i]);
}

/* =========================================================================
 * linear_weights / lw_series / parab_moments (rt_solvers_mod.f90:785-877)
 * ========================================================================= */
static const float LW_P[8] = {+5.000000000e-01f, -1.666666716e-01f, +4.166666791e-02f, -8.333330974e-03f,
                              +1.388740959e-03f, -1.983609400e-04f, +2.522676368e-05f, -2.834696488e-06f};
static const float PM_R[9] = {+3.333333433e-01f, -8.333329856e-02f, +1.666668802e-02f, -2.777901944e-03f,
                              +3.968053206e-04f, -4.948913192e-05f, +5.514686109e-06f, -5.894584660e-07f,
                              +5.153443894e-08f};

static inline float or_lw_series(float t)
{
  float p = fmaf(t, LW_P[7], LW_P[6]);
  for (int k = 5; k >= 0; k--) p = fmaf(t, p, LW_P[k]);
  return t * p;
}

static inline void lw32(float t, float *E, float *W, float *Psi, float *Esc)
{
  float u0;
  or_exp_neg1(t, E, &u0);
  float ut = u0 / t;
  float ps = or_lw_series(t);
  int thin = fabsf(t) <= 1.0f;
  *Psi = thin ? ps : 1.0f - ut;
  *Esc = thin ? 1.0f - ps : ut;
  *W = thin ? u0 - ps : ut - *E;
}

static inline void pm32(float t, float *E, float *U0, float *U1, float *q)
{
  or_exp_neg1(t, E, U0);
  *U1 = fabsf(t) <= 1.0f ? t * or_lw_series(t) : t - *U0;
  float p = fmaf(t, PM_R[8], PM_R[7]);
  for (int k = 6; k >= 0; k--) p = fmaf(t, p, PM_R[k]);
  float qs = (t * t) * p;
  *q = fabsf(t) <= 2.0f ? qs : t - 2.0f * (*U1 / t);
}

/* plain FP64 weights: exact exp/expm1, Taylor series where the forms cancel */
/* Taylor sums of the FP64 forms below |t| = 0.1, where the closed forms cancel:
 * Psi = sum_{k>=1} (-1)^(k+1) t^k/(k+1)!, U1 = sum_{k>=2} (-1)^k t^k/k!,
 * q = sum_{k>=3} 2 (-1)^(k+1) t^(k-1)/k!, each to 12 terms (truncation < 1e-17). */
static inline double series64(double t, int k0, int shift, double scale)
{
  /* sum_{k=k0}^{k0+11} scale (-1)^k t^(k-shift)/k!, Horner from the top */
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

static inline void lw64(double t, double *E, double *W, double *Psi, double *Esc)
{
  double tc = fmin(t, 700.0);
  *E = exp(-tc);
  double u0 = -expm1(-tc);
  if (fabs(t) < 0.1) {
    /* Psi = sum_{k>=2} (-1)^k t^(k-1)/k! */
    double ps = series64(t, 2, 1, 1.0);
    *Psi = ps;
    *Esc = 1.0 - ps;
    *W = u0 - ps;
  } else {
    double ut = u0 / t;
    *Psi = 1.0 - ut;
    *Esc = ut;
    *W = ut - *E;
  }
}

static inline void pm64(double t, double *E, double *U0, double *U1, double *q)
{
  double tc = fmin(t, 700.0);
  *E = exp(-tc);
  *U0 = -expm1(-tc);
  if (fabs(t) < 0.1) {
    *U1 = series64(t, 2, 0, 1.0);
    *q = series64(t, 3, 1, -2.0);
  } else {
    *U1 = t - *U0;
    *q = t - 2.0 * (*U1 / t);
  }
}

/* bezier3_weights (rt_solvers_mod.f90:1280-1304): the cubic-Bezier weights over
 * an interval of optical depth t, w_k = t int_0^1 b_k(u) exp(-t u) du with
 * b = u^3, 3u^2(1-u), 3u(1-u)^2, (1-u)^3.  For t <= 3 the series t E P3(-t),
 * t E P2(-t), t P2(t), t P3(t) with P2 = w2/t, P3 = w3/t the reference's own
 * relative-error minimax fits of degree 10 and 9 (b3_p2, b3_p3, :1305-1331);
 * above, the moments M_n = n M_(n-1) - t^n E from M0 = 1 - E, formed at
 * max(t, 3).  The a*b - c forms are fused. */
static const float B3_P2[11] = {+2.500000000e-01f, -1.000000238e-01f, +2.499995567e-02f, -4.761847202e-03f,
                                +7.440865738e-04f, -9.924791084e-05f, +1.156294547e-05f, -1.190877015e-06f,
                                +1.137804801e-07f, -1.100420821e-08f, +7.658396139e-10f};
static const float B3_P3[10] = {+2.500000000e-01f, -4.999998957e-02f, +8.333289996e-03f, -1.190488110e-03f,
                                +1.488493726e-04f, -1.653099389e-05f, +1.640762775e-06f, -1.503805294e-07f,
                                +1.414234507e-08f, -1.025371787e-09f};

static inline float or_b3_p2(float t)
{
  float p = fmaf(t, B3_P2[10], B3_P2[9]);
  for (int k = 8; k >= 0; k--) p = fmaf(t, p, B3_P2[k]);
  return p;
}
static inline float or_b3_p3(float t)
{
  float p = fmaf(t, B3_P3[9], B3_P3[8]);
  for (int k = 7; k >= 0; k--) p = fmaf(t, p, B3_P3[k]);
  return p;
}

static inline void bz32(float t, float *E, float *w0, float *w1, float *w2, float *w3)
{
  const float tser = 3.0f;
  float M0;
  or_exp_neg1(t, E, &M0);
  const float tb = fmaxf(t, tser);
  const float tb2 = tb * tb;
  const float tb3 = tb2 * tb;
  const float r3 = 1.0f / tb3;
  const float M1 = fmaf(-tb, *E, M0);
  const float M2 = fmaf(-tb2, *E, 2.0f * M1);
  const float M3 = fmaf(-tb3, *E, 3.0f * M2);
  const float b0 = M3 * r3;
  const float b1 = (3.0f * fmaf(M2, tb, -M3)) * r3;
  const float b2 = (3.0f * (fmaf(M1, tb2, -((2.0f * M2) * tb)) + M3)) * r3;
  const int ser = t <= tser;
  const float tE = t * *E;
  *w0 = ser ? tE * or_b3_p3(-t) : b0;
  *w1 = ser ? tE * or_b3_p2(-t) : b1;
  *w2 = ser ? t * or_b3_p2(t) : b2;
  *w3 = ser ? t * or_b3_p3(t) : ((M0 - b0) - b1) - b2;
}

void or_bezier3_weights_f32(int n, const float *t, float *w0, float *w1, float *w2, float *w3)
{
  for (int i = 0; i < n; i++) {
    float E;
    bz32(t[i], &E, &w0[i], &w1[i], &w2[i], &w3[i]);
  }
}

void or_linear_weights_f32(int n, const float *t, float *E, float *W, float *Psi, float *Esc)
{
  for (int i = 0; i < n; i++) lw32(t[i], &E[i], &W[i], &Psi[i], &Esc[i]);
}
void or_linear_weights_f64(int n, const double *t, double *E, double *W, double *Psi, double *Esc)
{
  for (int i = 0; i < n; i++) lw64(t[i], &E[i], &W[i], &Psi[i], &Esc[i]);
}
void or_parab_moments_f32(int n, const float *t, float *E, float *U0, float *U1, float *q)
{
  for (int i = 0; i < n; i++) pm32(t[i], &E[i], &U0[i], &U1[i], &q[i]);
}
void or_parab_moments_f64(int n, const double *t, double *E, double *U0, double *U1, double *q)
{
  for (int i = 0; i < n; i++) pm64(t[i], &E[i], &U0[i], &U1[i], &q[i]);
}

/* =========================================================================
 * Stencil (ray_mod.f90:493-512) and Keys cubic kernel (ray_mod.f90:581-597)
 * ========================================================================= */
static void cc_kernel(double s, double k[4])
{
  double s2 = s * s, s3 = s2 * s;
  k[0] = 0.5 * (-s3 + 2 * s2 - s);
  k[1] = 0.5 * (3 * s3 - 5 * s2 + 2);
  k[2] = 0.5 * (-3 * s3 + 4 * s2 + s);
  k[3] = 0.5 * (s3 - s2);
}

void or_set_stencil(const double ds[3], const double vec[3], double xkern[4], double ykern[4],
                    int *upo1, int *upo2, double *dsup)
{
  *dsup = ds[2] / fabs(vec[2]);
  double wt1 = -vec[0] / ds[0] * *dsup;
  double wt2 = -vec[1] / ds[1] * *dsup;
  double h1 = wt1 > 0 ? wt1 : wt1 + 1;
  double h2 = wt2 > 0 ? wt2 : wt2 + 1;
  *upo1 = wt1 > 0 ? -1 : -2;
  *upo2 = wt2 > 0 ? -1 : -2;
  cc_kernel(h1, xkern);
  cc_kernel(h2, ykern);
}

/* =========================================================================
 * QLG (HOP/qlg_mod.f90)
 * ========================================================================= */
#define QLG_NX 9019
static const float QLG_XSCL = 800.0f, QLG_RNX = 9019.0f;
static const float QLG_OVERPI = 0.3183098862f, QLG_GNORM = 0.4697186f, QLG_SQL2 = 0.8325546112f;
static const float QLG_RPI = 1.7724538509f, QLG_ISQPI = 0.5641895835f;

/* Weideman (1994) N = 32 rational coefficients, qlg_mod.f90:134-151 */
static const double W32_LD = 4.75682846001088411e+00;
static const double W32_AD[32] = {
    -1.30317978630500875e-12, +3.74107755472269789e-12, +8.03033538228436012e-12, -2.15435373143760700e-11,
    -5.54423561143486540e-11, +1.16582546820233235e-10, +4.15374271614691897e-10, -5.23102143724924582e-10,
    -3.20801514078875819e-09, +8.12488896568210460e-10, +2.37975567593842971e-08, +2.29304391194392872e-08,
    -1.48130789124396946e-07, -4.18407637053084035e-07, +4.25583313792292626e-07, +4.40153173159092505e-06,
    +6.82103194402497841e-06, -2.14096192018698432e-05, -1.30754492546239731e-04, -2.45329802700202065e-04,
    +3.92591360700705167e-04, +4.51954110534923473e-03, +1.90061557848454077e-02, +5.73044035298371918e-02,
    +1.40607162268937713e-01, +2.95444510715087261e-01, +5.46013972063934205e-01, +9.01925489364799993e-01,
    +1.34554416923454490e+00, +1.82566962963248147e+00, +2.26353729990026764e+00, +2.57225340812456960e+00};

/* Humlicek-Weideman fp64 hybrid, qlg_mod.f90:411-447 */
void or_qlg_ref_f64(double a, double v0, double dv, int n, double *K)
{
  const double ISQPI8 = 0.564189583547756287;
  double dr = W32_LD + a, nr0 = W32_LD - a;
  for (int f = 0; f < n; f++) {
    double v = v0 + (double)f * dv, av = fabs(v);
    if (av + a >= 15.0) {
      double tr = a * a - av * av + 0.5, ti = -2.0 * a * av;
      double q = 1.0 / (tr * tr + ti * ti);
      double ur = (a * tr + (-av) * ti) * q;
      K[f] = ISQPI8 * ur;
    } else {
      double di = -v;
      double q = 1.0 / (dr * dr + di * di);
      double zr = (nr0 * dr + v * di) * q, zi = (v * dr - nr0 * di) * q;
      double pr = W32_AD[0], pi_ = 0.0;
      for (int j = 1; j < 32; j++) {
        double t = pr * zr - pi_ * zi + W32_AD[j];
        pi_ = pr * zi + pi_ * zr;
        pr = t;
      }
      double ir = dr * q, ii = -di * q;
      double sr = ir * ir - ii * ii, si = 2.0 * ir * ii;
      K[f] = 2.0 * (pr * sr - pi_ * si) + ISQPI8 * ir;
    }
  }
}

/* Z_0.2(u)(1+u)^2, qlg_mod.f90:384-399 */
static double qlg_wr02(double u)
{
  const double A2 = 0.18741813853432507, GAM = 0.93709069267162530, KP = 0.81924853602069690;
  const double ETA = 0.14697983683153040, QRS = 0.16, DLN2 = 0.69314718055994531;
  double v = GAM * sqrt(u), L = 1.0 / (1.0 + u), G = exp(-DLN2 * u), Kv;
  or_qlg_ref_f64(A2, v, 0.0, 1, &Kv);
  double P = KP * (ETA * L + (1.0 - ETA) * G);
  return (Kv - P) / (QRS * KP) * (1.0 + u) * (1.0 + u);
}

/* qlg_init, qlg_mod.f90:364-375 */
void or_qlg_tables(float *tgx, float *th2x)
{
  for (int i = 0; i <= QLG_NX; i++) {
    double x = (double)i / 800.0;
    tgx[i] = (float)pow(2.0, -x * x);
    th2x[i] = (float)qlg_wr02(x * x);
  }
}

typedef struct { float ih, bL, gG, cZH, cL2; } qlg_coef_t;

/* bot_setup, qlg_mod.f90:538-554 */
static inline qlg_coef_t bot_setup(float gL, float D, float SQ, float S)
{
  qlg_coef_t c;
  float e = fmaf(gL, 0.60602209212341318f, D);
  c.ih = e / fmaf(gL, e, SQ);
  float r = gL * c.ih;
  float q = r * (1.0f - r);
  float sc = S * c.ih;
  float qs = q * sc;
  float x = 2.0f * r - 1.0f;
  c.bL = (QLG_OVERPI * r) * sc;
  c.gG = fmaf(qs, fmaf(x, -0.11019326278794868f, -0.064924393191013452f), (QLG_GNORM * (1.0f - r)) * sc);
  c.cZH = qs * fmaf(x, -0.10567135279610407f, 0.38494195930078284f);
  c.cL2 = qs * fmaf(x, 0.16241029253712097f, 0.04054415746208978f);
  return c;
}

/* qlg_bot_line_eval, qlg_mod.f90:556-571 */
static inline float bot_eval(const float *tgx, const float *th2x, const qlg_coef_t *c, float x)
{
  float xs = fabsf(x) * c->ih;
  float u = xs * xs;
  float L = 1.0f / (1.0f + u);
  /* nint(y) for y = min(xs*800, 9019) >= 0: y + 0.5f is exact or rounds to an
   * integer no larger than floor(y + 0.5) on [0.5, 9019], and every y below 0.5
   * (including the float just below, whose sum rounds up to 1) snaps to node 0;
   * written without lroundf so the point loop vectorises */
  const float y = fminf(xs * QLG_XSCL, QLG_RNX);
  const int ig = y < 0.5f ? 0 : (int)(y + 0.5f);
  float G = tgx[ig], W = th2x[ig];
  float p = fmaf(c->cZH, W, c->cL2);
  p = fmaf(L, p, c->bL);
  return fmaf(L, p, G * c->gG);
}

/* qlg_bot_coef / qlg_bot_eval (qlg_mod.f90:515-528): the split one-point form the
 * hydrogen profiles use, c[5] = (ih, bL, gG, cZH, cL2) */
void or_qlg_coef(float a, float c[5])
{
  qlg_coef_t k = bot_setup(a, 1.0f, QLG_SQL2, QLG_RPI);
  c[0] = k.ih;
  c[1] = k.bL;
  c[2] = k.gG;
  c[3] = k.cZH;
  c[4] = k.cL2;
}

float or_qlg_eval(const float *tgx, const float *th2x, const float c[5], float v)
{
  qlg_coef_t k = {c[0], c[1], c[2], c[3], c[4]};
  return bot_eval(tgx, th2x, &k, v) * QLG_ISQPI;
}

/* qlg_bot_sweep (qlg_mod.f90:222-257) = bot_setup(a, 1, SQL2, RPI) + eval */
void or_qlg_bot_sweep(const float *tgx, const float *th2x, float a, float v0, float dv, int n, float *K)
{
  qlg_coef_t c = bot_setup(a, 1.0f, QLG_SQL2, QLG_RPI);
  for (int f = 0; f < n; f++) K[f] = bot_eval(tgx, th2x, &c, fmaf((float)f, dv, v0));
}

/* qlg_bot_profile, qlg_mod.f90:682-689 */
void or_qlg_bot_profile(const float *tgx, const float *th2x, int n, const float *a, const float *q,
                        const float *vpr, const float *idf, float *h)
{
  for (int i = 0; i < n; i++) {
    float v = fabsf(q[i] - vpr[i]) * idf[i], K1;
    or_qlg_bot_sweep(tgx, th2x, a[i], v, 0.0f, 1, &K1);
    h[i] = ((K1 * QLG_ISQPI) * idf[i]) * (q[i] + 1.0f);
  }
}

/* qlg_bot_line (qlg_mod.f90:616-627): setup plus half-width */
typedef struct { float D, D2, SQ, D2h, D2G, D2L; } qlg_cell_t;
static inline qlg_cell_t bot_cell(float D)
{
  qlg_cell_t w;
  w.D = D;
  w.D2 = D * D;
  w.SQ = QLG_SQL2 * w.D2;
  w.D2h = 0.5f * w.D2;
  w.D2G = 1.5f * w.D2;
  w.D2L = 5.0f * w.D2;
  return w;
}

static inline float bot_halfwidth(const qlg_cell_t *w, float gL, float S, float ref, float lnq)
{
  float AL = ((QLG_OVERPI * gL) * S) / ref;
  float h1 = fmaf(w->D2, lnq, fminf(AL, w->D2G));
  float h2 = (AL - fmaxf(fmaf(gL, gL, -w->D2h), 0.0f)) + fminf(AL, w->D2L);
  return sqrtf(fmaxf(fmaxf(h1, h2), 0.0f));
}

/* qlg_bot_line_sweep, qlg_mod.f90:646-671; returns the number of K values */
static int line_sweep(const float *tgx, const float *th2x, const qlg_cell_t *w, float gL, float S,
                      float ref, float lnq, int nf, const double *llam, double llc, double pos,
                      double idl, float cap, int *fa, int *fb, float *hw, float *K)
{
  int ic = (int)lround(pos) + 1;
  int i1 = ic < 1 ? 1 : (ic > nf ? nf : ic);
  float x1 = (float)((llam[i1 - 1] - llc) * idl);
  qlg_coef_t c = bot_setup(gL, w->D, w->SQ, S);
  *hw = bot_halfwidth(w, gL, S, ref, lnq);
  int noff = (int)lroundf(fminf(fminf(*hw, cap), (float)(nf + abs(ic))));
  *fa = ic - noff > 1 ? ic - noff : 1;
  *fb = ic + noff < nf ? ic + noff : nf;
  if (*fa > *fb) return 0;
  float x0 = x1 - (float)(i1 - *fa);
  /* The last node's TGX is subnormal, and most window points of most lines snap to
   * it; its product with gG is the same for every such point, so it is formed once
   * per line (the same rounding), which keeps subnormal arithmetic -- microcoded
   * and a hundred times slower on x86 -- out of the point loop. */
  const float g_end = tgx[QLG_NX] * c.gG;
  /* That product is itself often a nonzero subnormal.  The last step at such points,
   * fma(L, p, g), is then taken on operands scaled by 2^64: exact scalings, so the
   * rounded result is the same whenever it is normal (else the direct form). */
  const int g_sub = g_end != 0.0f && fabsf(g_end) < FLT_MIN;
  const float g_big = g_end * 18446744073709551616.0f;      /* 2^64, exact */
  for (int f = 0; f <= *fb - *fa; f++) {
    const float x = x0 + (float)f;
    const float xs = fabsf(x) * c.ih;
    const float u = xs * xs;
    const float L = 1.0f / (1.0f + u);
    const float y = fminf(xs * QLG_XSCL, QLG_RNX);
    const int ig = y < 0.5f ? 0 : (int)(y + 0.5f);
    float p = fmaf(c.cZH, th2x[ig], c.cL2);
    p = fmaf(L, p, c.bL);
    if (ig == QLG_NX && g_sub) {
      const float k = fmaf(L, p * 18446744073709551616.0f, g_big) * 5.42101086242752217e-20f;  /* 2^-64 */
      K[f] = fabsf(k) >= FLT_MIN ? k : fmaf(L, p, g_end);
    } else {
      K[f] = fmaf(L, p, ig == QLG_NX ? g_end : tgx[ig] * c.gG);
    }
  }
  return *fb - *fa + 1;
}

int or_qlg_bot_line_sweep(const float *tgx, const float *th2x, float D, float gL, float S, float ref,
                          float lnq, int nf, const double *llam, double llc, double pos, double idl,
                          float cap, int *fa, int *fb, float *hw, float *K)
{
  qlg_cell_t w = bot_cell(D);
  return line_sweep(tgx, th2x, &w, gL, S, ref, lnq, nf, llam, llc, pos, idl, cap, fa, fb, hw, K);
}

/* lower_bound8 / upper_bound8 (linelist_mod.f90:1807-1844), 0-based: the first
 * index with a[i] >= x (n if none), the last index with a[i] <= x (-1 if none) */
static int lower_bound8(const double *a, int n, double x)
{
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (a[mid] >= x) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}
static int upper_bound8(const double *a, int n, double x)
{
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (a[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  return lo - 1;
}

int or_select_lines(const or_linelist_t *ll, int nf, const double *llam, float vmax, int *sel)
{
  int l0 = 0, l1 = ll->nline - 1, nsel = 0;
  double blue = 0, red = 0;
  if (ll->reach_in) {
    double hb1 = 0, hb2 = 0, rmax = 0;
    if (nf > 1) {
      hb1 = 0.5 * (llam[1] - llam[0]);
      hb2 = 0.5 * (llam[nf - 1] - llam[nf - 2]);
    }
    for (int l = 0; l < ll->nline; l++)
      if ((double)ll->reach_in[l] > rmax) rmax = ll->reach_in[l];
    blue = llam[0] - hb1 - (double)vmax;
    red = llam[nf - 1] + hb2 + (double)vmax;
    const int a = lower_bound8(ll->llam0, ll->nline, blue - rmax);
    const int b = upper_bound8(ll->llam0, ll->nline, red + rmax);
    l0 = a > l0 ? a : l0;
    l1 = b < l1 ? b : l1;
  }
  for (int l = l0; l <= l1; l++) {
    if (ll->active && !ll->active[l]) continue;
    if (ll->reach_in && (ll->llam0[l] + (double)ll->reach_in[l] < blue || ll->llam0[l] - (double)ll->reach_in[l] > red))
      continue;
    sel[nsel++] = l;
  }
  return nsel;
}

/* =========================================================================
 * add_opacity_equi (HOP/linelist_mod.f90:729-960), with or without per-line
 * reach (has_reach: select_lines, and lines centred beyond the chunk take the
 * unfloored reference at the nearer end and a window capped by their reach);
 * without the LTE scattering split (do_scat)
 * ========================================================================= */
int or_add_opacity_equi(const float *tgx, const float *th2x, const or_linelist_t *ll,
                        int nf, const double *llam, int ncell,
                        float *chi, float *eta, const float *cont, const float *logref,
                        const float *vproj, const float *inv_df, const float *vbar2, const float *e_kT,
                        const float *lnbase, const float *ne, const float *tothi, const float *stark_pe,
                        const float *dep_mem, int nlevel, int do_nlte, float tol, float line_reject_frac,
                        uint8_t *used, float *strength, float *reach)
{
  return or_add_opacity_equi_scat(tgx, th2x, ll, nf, llam, ncell, chi, eta, cont, logref, vproj, inv_df, vbar2,
                                  e_kT, lnbase, ne, tothi, stark_pe, dep_mem, nlevel, do_nlte, tol,
                                  line_reject_frac, used, strength, reach, NULL, NULL);
}

/* add_opacity_equi with line_scattering (do_scat, linelist_mod.f90:933-939): an LTE
 * line adds its profile to chi and eta and (1-eps) of it to chi_scat, in line order;
 * one_m_eps and chi_scat are (nf, ncell) like chi, NULL without do_scat. */
int or_add_opacity_equi_scat(const float *tgx, const float *th2x, const or_linelist_t *ll,
                             int nf, const double *llam, int ncell,
                             float *chi, float *eta, const float *cont, const float *logref,
                             const float *vproj, const float *inv_df, const float *vbar2, const float *e_kT,
                             const float *lnbase, const float *ne, const float *tothi, const float *stark_pe,
                             const float *dep_mem, int nlevel, int do_nlte, float tol, float line_reject_frac,
                             uint8_t *used, float *strength, float *reach, const float *one_m_eps,
                             float *chi_scat)
{
  const float ex_cutoff = -85.0f, voigt_peak = 0.5641895835f, sqrt_pi = 1.7724538509f;
  if (ll->nline == 0 || nf < 2) return 0;
  if (llam[nf - 1] < llam[0]) return 1;
  const double llam1 = llam[0];
  const double dllam = (llam[nf - 1] - llam[0]) / (double)(nf - 1);
  const double inv_dllam = 1.0 / dllam;
  const float sdl = (float)inv_dllam;
  const float flo_scale = fmaxf(tol, line_reject_frac) * tol;
  float *Kbuf = (float *)malloc(sizeof(float) * (size_t)nf);
  int *sel = (int *)malloc(sizeof(int) * (size_t)(ll->nline > 0 ? ll->nline : 1));
  float vmax = 0.0f;
  if (ll->reach_in)
    for (int i = 0; i < ncell; i++) vmax = fmaxf(vmax, fabsf(vproj[i]));
  const int nsel = or_select_lines(ll, nf, llam, vmax, sel);
  for (int i = 0; i < ncell; i++) {
    float *ch = chi + (size_t)nf * i, *et = eta + (size_t)nf * i;
    const float *co = cont + (size_t)nf * i, *lr = logref + (size_t)nf * i;
    int f0_prev = -1;
    float refl_c = 0, lref_c = 0;
    const float idf = inv_df[i];
    qlg_cell_t qw = bot_cell(sdl / idf);
    const float lvb2 = or_logf1(vbar2[i]);
    const float unsold_c = or_exp4(0.3f * lvb2) * tothi[i];
    const float ekt = e_kT[i], ne_c = ne[i], tothi_c = tothi[i], starkpe = stark_pe[i];
    const float vproj_c = vproj[i];
    const float base = lnbase[i];
    for (int isel = 0; isel < nsel; isel++) {
      const int l = sel[isel];
      double llc = ll->llam0[l] - (double)vproj_c;
      double pos = (llc - llam1) * inv_dllam;
      int f0 = (int)lround(pos) + 1;
      f0 = f0 < 1 ? 1 : (f0 > nf ? nf : f0);
      float ex = ll->lower_ev[l] * ekt;
      float arg = (base + ll->gpref[l]) - ex;
      if (arg < ex_cutoff) continue;
      const int outside = ll->reach_in && (llc < llam[0] || llc > llam[nf - 1]);
      float Rij, ref, lref_o = 0.0f;
      int fe = 0;
      if (outside) {
        /* centred beyond the chunk: the reference at the nearer end, unfloored */
        fe = llc < llam[0] ? 1 : nf;
        lref_o = lr[fe - 1];
        if (arg <= lref_o) continue;
        Rij = or_exp4(arg);
        ref = tol * co[fe - 1];
      } else {
        if (f0 != f0_prev) {
          f0_prev = f0;
          refl_c = tol * co[f0 - 1];
          float flo = flo_scale * ch[f0 - 1];
          if (flo > refl_c) {
            refl_c = flo;
            lref_c = or_logf1(flo * sqrt_pi);
          } else {
            lref_c = lr[f0 - 1];
          }
        }
        if (arg <= lref_c) continue;
        Rij = or_exp4(arg);
        ref = refl_c;
        if (voigt_peak * Rij <= ref) continue;
      }
      int nlte = do_nlte && ll->lev_i && ll->lev_j && ll->lev_i[l] > 0 && ll->lev_j[l] > 0;
      float bi = 1.0f, bj = 1.0f;
      if (nlte) {
        bi = dep_mem[(size_t)i + (size_t)ncell * (ll->lev_i[l] - 1)];
        bj = dep_mem[(size_t)i + (size_t)ncell * (ll->lev_j[l] - 1)];
      }
      float a = ll->grad[l];
      if (ll->unsold[l]) a = fmaf(ll->gw1[l], unsold_c, a);
      else a = fmaf(ll->gw1[l] * or_exp4(ll->gw2[l] * lvb2), tothi_c, a);
      if (ll->gstk[l] >= 0.0f) a = fmaf(ll->gstk[l], ne_c, a);
      else a = fmaf(-ll->gstk[l], starkpe, a);
      a = a * sdl;
      float cap = FLT_MAX, lnq;
      if (outside) {
        cap = (float)((double)ll->reach_in[l] * inv_dllam);
        lnq = arg - lref_o;
      } else {
        if (strength) {
          float st = (voigt_peak * Rij) / co[f0 - 1];
          if (st > strength[l]) strength[l] = st;
        }
        lnq = arg - lref_c;
      }
      int fa, fb;
      float hw;
      int nk = line_sweep(tgx, th2x, &qw, a, Rij * qw.D, ref, lnq, nf, llam, llc, pos, inv_dllam,
                          cap, &fa, &fb, &hw, Kbuf);
      if (reach) {
        float rch = (float)((double)hw * dllam);
        if (rch > reach[l]) reach[l] = rch;
      }
      if (nk == 0) continue;
      if (used) used[l] = 1;
      if (chi_scat && !nlte) {
        float *cs = chi_scat + (size_t)nf * i;
        const float *om = one_m_eps + (size_t)nf * i;
        for (int f = fa; f <= fb; f++) {
          float lte = Kbuf[f - fa];
          ch[f - 1] = ch[f - 1] + lte;
          et[f - 1] = et[f - 1] + lte;
          cs[f - 1] = fmaf(om[f - 1], lte, cs[f - 1]);
        }
      } else {
        for (int f = fa; f <= fb; f++) {
          float lte = Kbuf[f - fa];
          ch[f - 1] = fmaf(lte, bi, ch[f - 1]);
          et[f - 1] = fmaf(lte, bj, et[f - 1]);
        }
      }
      f0_prev = -1;
    }
  }
  free(Kbuf);
  free(sel);
  return 0;
}

/* =========================================================================
 * The plain FP64 path of the LTE pass's line opacity: add_opacity_equi
 * (HOP/linelist_mod.f90:729-960) and the QLG-bot profile (qlg_mod.f90:538-671)
 * step for step in double.  The tables are qlg_init's formulas in fp64 (not
 * rounded to float), the fitted float constants are the exact values they stand
 * for (1/pi, sqrt(ln2/pi), sqrt(ln2), 1/sqrt(pi)), exp and log are libm's double
 * functions, and the Doppler shift, the tolerance references and xhat are double.
 * No line selection by reach, no NLTE departures, no scattering split.
 * ========================================================================= */
void or_qlg_tables_f64(double *tgx, double *th2x)
{
  for (int i = 0; i <= QLG_NX; i++) {
    double x = (double)i / 800.0;
    tgx[i] = pow(2.0, -x * x);
    th2x[i] = qlg_wr02(x * x);
  }
}

typedef struct { double ih, bL, gG, cZH, cL2; } qlg_coef64_t;

static qlg_coef64_t bot_setup64(double gL, double D, double SQ, double S)
{
  qlg_coef64_t c;
  double e = fma(gL, 0.60602209212341318, D);
  c.ih = e / fma(gL, e, SQ);
  double r = gL * c.ih;
  double q = r * (1.0 - r);
  double sc = S * c.ih;
  double qs = q * sc;
  double x = 2.0 * r - 1.0;
  c.bL = (0.31830988618379067 * r) * sc;
  c.gG = fma(qs, fma(x, -0.11019326278794868, -0.064924393191013452), (0.46971863934982566 * (1.0 - r)) * sc);
  c.cZH = qs * fma(x, -0.10567135279610407, 0.38494195930078284);
  c.cL2 = qs * fma(x, 0.16241029253712097, 0.04054415746208978);
  return c;
}

static double bot_eval64(const double *tgx, const double *th2x, const qlg_coef64_t *c, double x)
{
  double xs = fabs(x) * c->ih;
  double u = xs * xs;
  double L = 1.0 / (1.0 + u);
  int ig = (int)lround(fmin(xs * 800.0, 9019.0));
  double p = fma(c->cZH, th2x[ig], c->cL2);
  p = fma(L, p, c->bL);
  return fma(L, p, tgx[ig] * c->gG);
}

/* chl (nf, ncell) accumulated in place for one species; xhat (nf, ncell) in double */
int or_opacity_f64(const double *tgx, const double *th2x, const or_linelist_t *ll, int nf, const double *llam,
                   int ncell, double *chl, const double *xhat, const double *vproj, const float *inv_df,
                   const float *vbar2, const float *e_kT, const float *lnbase, const float *ne, const float *tothi,
                   const float *stark_pe, double tol)
{
  const double ex_cutoff = -85.0, voigt_peak = 0.56418958354775628, sqrt_pi = 1.7724538509055160;
  if (ll->nline == 0 || nf < 2) return 0;
  if (llam[nf - 1] < llam[0]) return 1;
  const double llam1 = llam[0];
  const double dllam = (llam[nf - 1] - llam[0]) / (double)(nf - 1);
  const double inv_dllam = 1.0 / dllam;
  const double sdl = inv_dllam;
  const float tolf = (float)tol;
  const double flo_scale = (double)(tolf * tolf);
  const double lt = log(tol / voigt_peak);
  for (int i = 0; i < ncell; i++) {
    double *ch = chl + (size_t)nf * i;
    const double *xh = xhat + (size_t)nf * i;
    const double D = sdl / (double)inv_df[i], D2 = D * D, SQ = 0.83255461115769776 * D2;
    const double lvb2 = log((double)vbar2[i]);
    const double unsold_c = exp(0.3 * lvb2) * (double)tothi[i];
    const double ekt = e_kT[i], ne_c = ne[i], tothi_c = tothi[i], starkpe = stark_pe[i], base = lnbase[i];
    for (int l = 0; l < ll->nline; l++) {
      if (ll->active && !ll->active[l]) continue;
      const double llc = ll->llam0[l] - vproj[i];
      const double pos = (llc - llam1) * inv_dllam;
      const int ic = (int)lround(pos) + 1;
      const int f0 = ic < 1 ? 1 : (ic > nf ? nf : ic);
      const double arg = (base + (double)ll->gpref[l]) - (double)ll->lower_ev[l] * ekt;
      if (arg < ex_cutoff) continue;
      const double cont0 = xh[f0 - 1];
      double refl = tol * cont0, lref;
      const double flo = flo_scale * ch[f0 - 1];
      if (flo > refl) {
        refl = flo;
        lref = log(flo * sqrt_pi);
      } else {
        lref = cont0 > 0.0 ? lt + log(cont0) : -DBL_MAX;
      }
      if (arg <= lref) continue;
      const double Rij = exp(arg);
      if (voigt_peak * Rij <= refl) continue;
      double a = ll->grad[l];
      const double gw1 = ll->gw1[l];
      if (ll->unsold[l]) a = fma(gw1, unsold_c, a);
      else if (gw1 != 0.0) a = fma(gw1 * exp((double)ll->gw2[l] * lvb2), tothi_c, a);
      const double gs = ll->gstk[l];
      a = gs >= 0.0 ? fma(gs, ne_c, a) : fma(-gs, starkpe, a);
      a *= sdl;
      const double S = Rij * D;
      const double x1 = (llam[f0 - 1] - llc) * inv_dllam;
      const qlg_coef64_t c = bot_setup64(a, D, SQ, S);
      const double AL = ((0.31830988618379067 * a) * S) / refl;
      const double h1 = fma(D2, arg - lref, fmin(AL, 1.5 * D2));
      const double h2 = (AL - fmax(fma(a, a, -0.5 * D2), 0.0)) + fmin(AL, 5.0 * D2);
      const double hw = sqrt(fmax(fmax(h1, h2), 0.0));
      const int noff = (int)lround(fmin(hw, (double)(nf + abs(ic))));
      const int fa = ic - noff > 1 ? ic - noff : 1;
      const int fb = ic + noff < nf ? ic + noff : nf;
      if (fa > fb) continue;
      const double x0 = x1 - (double)(f0 - fa);
      for (int f = fa; f <= fb; f++) ch[f - 1] += bot_eval64(tgx, th2x, &c, x0 + (double)(f - fa));
    }
  }
  return 0;
}

/* =========================================================================
 * Background and work units
 * ========================================================================= */
/* lte_background_opacities (rt_patch_mod.f90:2004-2023): beta, Bnu */
void or_lte_background(int nf, int ncell, const double *nu, const float *temp, float *beta, float *Bnu)
{
  for (int i = 0; i < ncell; i++) {
    float h_kT = (float)(OR_H_K / (double)temp[i]);
    for (int f = 0; f < nf; f++) {
      float hv = (float)(nu[f] * (double)h_kT), E, u0;
      or_exp_neg1(hv, &E, &u0);
      float b = fmaxf(E, FLT_MIN);
      beta[(size_t)f + (size_t)nf * i] = b;
      Bnu[(size_t)f + (size_t)nf * i] = b / (1.0f - b);
    }
  }
}

/* lte_background_emission with sigma = 0 (eta = chi_c Bnu, rt_patch_mod.f90:2309-2326)
 * then convert_to_work_units (rt_patch_mod.f90:3518-3536): xhat = chi + eta,
 * ehat = eta/beta.  chi_c is per cell (frequency independent grey continuum). */
void or_lte_work(int nf, int ncell, const float *chi_c, const float *beta, const float *Bnu,
                 float *xhat, float *ehat)
{
  for (int i = 0; i < ncell; i++)
    for (int f = 0; f < nf; f++) {
      size_t k = (size_t)f + (size_t)nf * i;
      float etav = chi_c[i] * Bnu[k];
      xhat[k] = chi_c[i] + etav;
      ehat[k] = etav / beta[k];
    }
}

/* logref of add_linelist_opacities (composition_mod.f90:1766-1772) */
void or_logref(int n, const float *xhat, float tol, float *logref)
{
  const float voigt_peak = 0.5641895835f;
  const float lt = or_logf1(tol / voigt_peak);
  for (int i = 0; i < n; i++) logref[i] = xhat[i] > 0.0f ? lt + or_logf1(xhat[i]) : -FLT_MAX;
}

/* work_to_transfer_units without split rates or line scattering
 * (rt_patch_mod.f90:3571-3651); returns the number of floored points */
int or_work_to_transfer_units(int nf, int ncell, float *w1, float *w2, const float *beta,
                              double maser_chi_floor, int suppress_masers)
{
  int nfl = 0;
  const float fl = (float)maser_chi_floor;
  for (size_t k = 0; k < (size_t)nf * ncell; k++) {
    float xhat = w1[k];
    float etav = w2[k] * beta[k];
    float chi = xhat - etav;
    float floor_ = fmaxf(fl * fabsf(xhat), FLT_MIN);
    if (suppress_masers) chi = fmaxf(chi, floor_);
    else if (fabsf(chi) < floor_) { chi = copysignf(floor_, chi); nfl++; }
    w1[k] = chi;
    w2[k] = etav / chi;
  }
  return nfl;
}

/* integrate_intensity (rt_patch_mod.f90:3399-3431) */
void or_integrate_intensity(int nf, int ncell, float wmu, const float *work3, const float *psi,
                            float *Jnu, float *PsiJ)
{
  float w2 = 2.0f * wmu;
  for (size_t k = 0; k < (size_t)nf * ncell; k++) {
    Jnu[k] = fmaf(w2, work3[k], Jnu[k]);
    if (psi && PsiJ) PsiJ[k] = fmaf(w2, psi[k], PsiJ[k]);
  }
}

/* save_intensity (rt_patch_mod.f90:4151-4208): ie = <I>_xy 2h nu^5/(c^3 AA),
 * flux = 2 pi sum_mu wmu ie.  I_top is (nf, nx, ny, nmu). */
void or_save_intensity(int nf, int nx, int ny, int nmu, const double *nu, const float *I_top,
                       const double *wmu, float *ie, float *flux)
{
  const double conversion = 2.0 * OR_HH / (OR_CC * OR_CC * OR_CC * OR_CM_TO_AA);
  for (int f = 0; f < nf; f++) flux[f] = 0.0f;
  for (int mu = 0; mu < nmu; mu++) {
    for (int f = 0; f < nf; f++) {
      double n5 = nu[f] * nu[f] * nu[f] * nu[f] * nu[f];
      float acc = 0.0f;
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          float i3 = (float)(conversion * n5 * (double)I_top[(size_t)f + (size_t)nf * ((size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * mu))]);
          acc += i3;
        }
      ie[(size_t)f + (size_t)nf * mu] = acc / (float)(nx * ny);
    }
  }
  for (int mu = 0; mu < nmu; mu++) {
    float w = (float)(2.0 * OR_PI * wmu[mu]);
    for (int f = 0; f < nf; f++) flux[f] = fmaf(w, ie[(size_t)f + (size_t)nf * mu], flux[f]);
  }
}

/* =========================================================================
 * Formal solvers, rotate_array and boundaries for REAL = float and double
 * ========================================================================= */
static inline float tiny_f32(void) { return FLT_MIN; }
static inline float huge_f32(void) { return FLT_MAX; }
static inline double tiny_f64(void) { return DBL_MIN; }
static inline double huge_f64(void) { return DBL_MAX; }

#define REAL float
#define SFX(n) n##_f32
#define FMA fmaf
#define RABS fabsf
#define RMAX fmaxf
#define RMIN fminf
#define RCOPYSIGN copysignf
#define LW lw32
#define PM pm32
#include "or_solvers.inc"
#undef REAL
#undef SFX
#undef FMA
#undef RABS
#undef RMAX
#undef RMIN
#undef RCOPYSIGN
#undef LW
#undef PM

#define REAL double
#define SFX(n) n##_f64
#define FMA fma
#define RABS fabs
#define RMAX fmax
#define RMIN fmin
#define RCOPYSIGN copysign
#define LW lw64
#define PM pm64
#include "or_solvers.inc"

/* =========================================================================
 * long_char_hermite (rt_solvers_mod.f90:1052-1504), fp32: the chain-rule
 * cubic-Hermite long characteristics.  dchi/ds by chi = (chi/Pe) Pe and dS/dtau
 * by S = rho Bnu from parabolas through three samples (herm_dtau, herm_source),
 * cubic-Bezier weights (bezier3_weights), the monotone clamp of the control
 * points.  The first plane starts from the upstream ghost: with its
 * thermodynamic state given (the bottom's ghost model or an upstream
 * neighbour) the full step, else the zeroed top ghost's secant step
 * (herm_first).  Slabs of at least 3 planes (the third parabola sample is then
 * always a plane of the slab).  The a*b + c forms are fused as listed.
 * ========================================================================= */
typedef struct {
  float rdsup, dsup1, dsup2, dtmax, Imax;
  int get_rates;
} or_herm_c;

static float herm_dtau(const or_herm_c *K, float xxup, float xxc, float xx3, float peu, float rpeu, float gpu,
                       float pec, float rpec, float gpc, float rpe3, int center)
{
  const float dtmin = 1e-20f;
  const float hh = 0.5f * K->rdsup;
  const float t1 = (xxc - xxup) * K->rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpu = xxup * rpeu, rxpc = xxc * rpec, rxp3 = xx3 * rpe3;
  float drxpu, drxpc;
  if (center) {
    drxpc = (rxp3 - rxpu) * hh;
    drxpu = (fmaf(-3.0f, rxpu, 4.0f * rxpc) - rxp3) * hh;
  } else {
    drxpu = (rxpc - rxp3) * hh;
    drxpc = fmaf(3.0f, rxpc, fmaf(-4.0f, rxpu, rxp3)) * hh;
  }
  float mup = fmaf(rxpu, gpu, peu * drxpu);
  float mc = fmaf(rxpc, gpc, pec * drxpc);
  mup = sgn * fmaxf(0.0f, fminf(sgn * mup, 2.0f * fabsf(t1)));
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 2.0f * fabsf(t1)));
  float dt = fmaf(K->dsup1, xxup + xxc, K->dsup2 * (mup - mc));
  dt = fmaxf(copysignf(fmaxf(fabsf(dt), dtmin), dt), K->dtmax);
  return dt;
}

static void herm_source(const or_herm_c *K, float xxup, float xxc, float ssup, float ssc, float ss3, float betau,
                        float betac, float beta3, float hk, float Inuup, float aTu, float aTc, int center, float dt,
                        float ex, float w0, float w1, float w2, float w3, float *Inu, float *plam)
{
  const float third = 0.333333343f;
  const float hh = 0.5f * K->rdsup;
  const float r1mbu = 1.0f / (1.0f - betau), r1mbc = 1.0f / (1.0f - betac), r1mb3 = 1.0f / (1.0f - beta3);
  const float Bu = betau * r1mbu, Bc = betac * r1mbc, B3 = beta3 * r1mb3;
  const float rhou = ssup / Bu, rhoc = ssc / Bc, rho3 = ss3 / B3;
  float drhu, drhc;
  if (center) {
    drhc = (rho3 - rhou) * hh;
    drhu = (fmaf(-3.0f, rhou, 4.0f * rhoc) - rho3) * hh;
  } else {
    drhu = (rhoc - rho3) * hh;
    drhc = fmaf(3.0f, rhoc, fmaf(-4.0f, rhou, rho3)) * hh;
  }
  const float rxxu = 1.0f / xxup, rxxc = 1.0f / xxc;
  const float gu = ((hk * r1mbu) * aTu) * rxxu;
  const float gc = ((hk * r1mbc) * aTc) * rxxc;
  const float dt3 = dt * third;
  float P1 = fmaf(dt3, fmaf(ssup, gu, (Bu * drhu) * rxxu), ssup);
  float P2 = fmaf(-dt3, fmaf(ssc, gc, (Bc * drhc) * rxxc), ssc);
  const float smin = fminf(ssup, ssc), smax = fmaxf(ssup, ssc);
  P1 = fminf(fmaxf(P1, smin), smax);
  P2 = fminf(fmaxf(P2, smin), smax);
  float I = fmaf(w3, ssc, fmaf(w2, P2, fmaf(w1, P1, fmaf(w0, ssup, Inuup * ex))));
  *Inu = fmaxf(-K->Imax, fminf(K->Imax, I));
  const float d1 = fminf(fmaxf((Bu * third) / Bc, 0.0f), 1.0f);
  const float d2 = fminf(fmaxf(fmaf(-dt3, gc, 0.666666687f), 0.0f), 1.0f);
  *plam = (K->get_rates && dt > 0 && xxc > 0) ? (fmaf(w1, d1, w2 * d2) + w3) * rxxc : 0.0f;
}

static void herm_first(const or_herm_c *K, float xxup, float xxc, float xxdn, float ssup, float ssc, float ssdn,
                       float betac, float betadn, float hk, float Inuup, float pec, float rpec, float rpedn,
                       float gpc, float aTc, float *Inu, float *plam)
{
  const float dtmin = 1e-20f, third = 0.333333343f;
  const float t1 = (xxc - xxup) * K->rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpc = xxc * rpec;
  float mc = fmaf(rxpc, gpc, (pec * fmaf(xxdn, rpedn, -rxpc)) * K->rdsup);
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 2.0f * fabsf(t1)));
  float dt = fmaf(K->dsup1, xxup + xxc, K->dsup2 * (t1 - mc));
  dt = fmaxf(copysignf(fmaxf(fabsf(dt), dtmin), dt), K->dtmax);
  float ex, w0, w1, w2, w3;
  bz32(dt, &ex, &w0, &w1, &w2, &w3);
  const float r1mbc = 1.0f / (1.0f - betac), r1mbdn = 1.0f / (1.0f - betadn);
  const float Bc = betac * r1mbc, Bdn = betadn * r1mbdn;
  const float Gc = ((hk * r1mbc) * aTc) / xxc;
  const float rhoc = ssc / Bc, rhodn = ssdn / Bdn;
  float taudn = K->dsup1 * (xxc + xxdn);
  taudn = copysignf(fmaxf(fabsf(taudn), dtmin), taudn);
  const float dSc = fmaf(ssc, Gc, (Bc * (rhodn - rhoc)) / taudn);
  const float dSu = (ssc - ssup) / dt;
  const float dt3 = dt * third;
  float P1 = fmaf(dt3, dSu, ssup);
  float P2 = fmaf(-dt3, dSc, ssc);
  const float smin = fminf(ssup, ssc), smax = fmaxf(ssup, ssc);
  P1 = fminf(fmaxf(P1, smin), smax);
  P2 = fminf(fmaxf(P2, smin), smax);
  float I = fmaf(w3, ssc, fmaf(w2, P2, fmaf(w1, P1, fmaf(w0, ssup, Inuup * ex))));
  *Inu = fmaxf(-K->Imax, fminf(K->Imax, I));
  *plam = (K->get_rates && dt > 0 && xxc > 0) ? (fmaf(w1, third, w2) + w3) / xxc : 0.0f;
}

/* work (nf, nx, ny, 0:nz+1, 3) with the upstream ghost plane already set; beta
 * (nf, nx, ny, nz); pe, dpe_dz, dlnt_dz, temp (nx, ny, nz); hknu (nf) = h/k nu;
 * g_* (nx, ny) the ghost's thermodynamics, all NULL for the zeroed top ghost;
 * gfac = dir |mu| / (code length) converts the d/dz to d/ds along the ray. */
int or_long_char_hermite(const or_slab_t *s, float *work, float *psi, const float *beta, const float *pe,
                         const float *dpe_dz, const float *dlnt_dz, const float *temp, const float *hknu,
                         const float *g_pe, const float *g_dpe_dz, const float *g_dlnt_dz, const float *g_temp,
                         double code_length)
{
  const int nf = s->nf, nx = s->nx, ny = s->ny, nz = s->nz, dir = s->dir;
  if (nz < 3) return 1;
  const float ds = (float)(s->ds[2]);
  const float dsup = (float)((double)ds / fabs(s->vec[2]));
  or_herm_c K;
  K.rdsup = 1.0f / dsup;
  K.dsup1 = 0.5f * dsup;
  K.dsup2 = (0.0833333358f * dsup) * dsup;
  K.dtmax = -(float)s->maser_dtau_max;
  K.Imax = (float)s->maser_Inu_max;
  K.get_rates = s->get_psi;
  const float gfac = (float)((double)dir * fabs(s->vec[2]) / code_length);
  const int ghost_thermo = g_pe != NULL;
  const int zs = dir > 0 ? 1 : nz, ze = dir > 0 ? nz : 1;
#define HW(f, x, y, z, k) ((size_t)(f) + (size_t)nf * ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * ((size_t)(z) + (size_t)(nz + 2) * (size_t)(k)))))
#define HP(f, x, y, z) ((size_t)(f) + (size_t)nf * ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * (size_t)((z) - 1))))
#define HC(x, y, z) ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * (size_t)((z) - 1)))
  for (int z = zs; dir > 0 ? z <= ze : z >= ze; z += dir) {
    const int zup = z - dir;
    const int first = z == zs, last = z == ze;
    const int center = !last;
    const int zt = last ? ze - 2 * dir : z + dir;
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        const float pec = pe[HC(x, y, z)], rpec = 1.0f / pec;
        const float gpc = gfac * dpe_dz[HC(x, y, z)];
        const float aTc = (gfac * dlnt_dz[HC(x, y, z)]) / temp[HC(x, y, z)];
        if (first && !ghost_thermo) {
          const int zdn = z + dir;
          const float rpedn = 1.0f / pe[HC(x, y, zdn)];
          for (int f = 0; f < nf; f++) {
            float I, pl;
            herm_first(&K, work[HW(f, x, y, zup, 0)], work[HW(f, x, y, z, 0)], work[HW(f, x, y, zdn, 0)],
                       work[HW(f, x, y, zup, 1)], work[HW(f, x, y, z, 1)], work[HW(f, x, y, zdn, 1)],
                       beta[HP(f, x, y, z)], beta[HP(f, x, y, zdn)], hknu[f], work[HW(f, x, y, zup, 2)], pec, rpec,
                       rpedn, gpc, aTc, &I, &pl);
            work[HW(f, x, y, z, 2)] = I;
            if (psi && K.get_rates) psi[HP(f, x, y, z)] = pl;
          }
          continue;
        }
        float peu, rpeu, gpu, aTu, rTup = 0.0f;
        if (first) {
          peu = g_pe[x + (size_t)nx * y];
          rpeu = 1.0f / peu;
          gpu = gfac * g_dpe_dz[x + (size_t)nx * y];
          rTup = 1.0f / g_temp[x + (size_t)nx * y];
          aTu = (gfac * g_dlnt_dz[x + (size_t)nx * y]) * rTup;
        } else {
          peu = pe[HC(x, y, zup)];
          rpeu = 1.0f / peu;
          gpu = gfac * dpe_dz[HC(x, y, zup)];
          aTu = (gfac * dlnt_dz[HC(x, y, zup)]) / temp[HC(x, y, zup)];
        }
        const float rpet = 1.0f / pe[HC(x, y, zt)];
        for (int f = 0; f < nf; f++) {
          const float bu = first ? fmaxf(or_exp4(-(hknu[f] * rTup)), FLT_MIN) : beta[HP(f, x, y, zup)];
          const float xxup = work[HW(f, x, y, zup, 0)], xxc = work[HW(f, x, y, z, 0)];
          const float dt = herm_dtau(&K, xxup, xxc, work[HW(f, x, y, zt, 0)], peu, rpeu, gpu, pec, rpec, gpc, rpet,
                                     center);
          float ex, w0, w1, w2, w3;
          bz32(dt, &ex, &w0, &w1, &w2, &w3);
          float I, pl;
          herm_source(&K, xxup, xxc, work[HW(f, x, y, zup, 1)], work[HW(f, x, y, z, 1)], work[HW(f, x, y, zt, 1)], bu,
                      beta[HP(f, x, y, z)], beta[HP(f, x, y, zt)], hknu[f], work[HW(f, x, y, zup, 2)], aTu, aTc,
                      center, dt, ex, w0, w1, w2, w3, &I, &pl);
          work[HW(f, x, y, z, 2)] = I;
          if (psi && K.get_rates) psi[HP(f, x, y, z)] = pl;
        }
      }
  }
#undef HW
#undef HP
#undef HC
  return 0;
}

/* =========================================================================
 * long_char_hermite2 (rt_solvers_mod.f90:1536-1895), fp32 with the reference's
 * real(8) dtau, 1/dtau and weights: the hybrid solver.  dtau as herm_dtau with
 * the control-point bound |dchi/ds| <= 3 |secant| (herm2_step :1758-1862);
 * the source is long_char_quadratic's parabola, dS/dtau at the target MC-limited
 * from the secants of the two intervals beside it (the second interval's dtau by
 * the same chain rule), on the last plane the backward one-sided difference over
 * (two-up, up, target) clamped to 2 |secant| when that sample is a plane of the
 * slab, else the interval secant.  herm2_first (:1869-1894) is the zeroed top
 * ghost's step.  Slabs of at least 2 planes.  ghost: 0 the zeroed top ghost,
 * 1 an upstream neighbour's exit plane, 2 the bottom's ghost model; 1 and 2
 * differ only for nz == 2 (the last plane's third-sample Pe, :1704-1709).
 * ========================================================================= */
typedef struct {
  float rdsup, dsup1, dsup2, Imax;
  double dtmax;
  int get_rates;
} or_herm2_c;

static double herm2_clamp(double dt, double dtmax)
{
  return fmax(copysign(fmax(fabs(dt), (double)1e-20f), dt), dtmax);
}

static void herm2_weights(const or_herm2_c *K, double dt, double rdt, float ex, float U0, float U1, float q,
                          float xxc, float ssup, float ssc, float dsdtau, float Inuup, float *Inu, float *plam)
{
  const double B = (2.0 * (double)U1 - (double)q) * rdt;
  const double A = (double)U0 - B;
  const float C = q - U1;
  const float I = fmaf(C, dsdtau, fmaf((float)B, ssc, fmaf((float)A, ssup, Inuup * ex)));
  *Inu = fmaxf(-K->Imax, fminf(K->Imax, I));
  *plam = (K->get_rates && dt > 0 && xxc > 0) ? (float)B / xxc : 0.0f;
}

static void herm2_step(const or_herm2_c *K, float xxup, float xxc, float xx3, float ssup, float ssc, float ss3,
                       float Inuup, float peu, float rpeu, float gpu, float pec, float rpec, float gpc, float pe3,
                       float rpe3, float gp3, int center, int onesided, float *Inu, float *plam)
{
  const float hh = 0.5f * K->rdsup;
  const float t1 = (xxc - xxup) * K->rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpu = xxup * rpeu, rxpc = xxc * rpec, rxp3 = xx3 * rpe3;
  float drxpu, drxpc;
  if (center) {
    drxpc = (rxp3 - rxpu) * hh;
    drxpu = (fmaf(-3.0f, rxpu, 4.0f * rxpc) - rxp3) * hh;
  } else {
    drxpu = (rxpc - rxp3) * hh;
    drxpc = fmaf(3.0f, rxpc, fmaf(-4.0f, rxpu, rxp3)) * hh;
  }
  float mup = fmaf(rxpu, gpu, peu * drxpu);
  float mc = fmaf(rxpc, gpc, pec * drxpc);
  mup = sgn * fmaxf(0.0f, fminf(sgn * mup, 3.0f * fabsf(t1)));
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 3.0f * fabsf(t1)));
  const double dt = herm2_clamp((double)fmaf(K->dsup1, xxup + xxc, K->dsup2 * (mup - mc)), K->dtmax);
  const double rdt = 1.0 / dt;
  float ex, U0, U1, q;
  pm32((float)dt, &ex, &U0, &U1, &q);
  const float s1 = (ssc - ssup) * (float)rdt;
  float dsdtau = s1;
  if (center) {
    const float t3 = (xx3 - xxc) * K->rdsup;
    const float sgn3 = copysignf(1.0f, t3);
    const float drxp3 = fmaf(3.0f, rxp3, fmaf(-4.0f, rxpc, rxpu)) * hh;
    float m3 = fmaf(rxp3, gp3, pe3 * drxp3);
    m3 = sgn3 * fmaxf(0.0f, fminf(sgn3 * m3, 3.0f * fabsf(t3)));
    const double dt3 = herm2_clamp((double)fmaf(K->dsup1, xxc + xx3, K->dsup2 * (mc - m3)), K->dtmax);
    const float s3 = (ss3 - ssc) / (float)dt3;
    const float avg = 0.5f * (s1 + s3);
    dsdtau = (copysignf(1.0f, s1) + copysignf(1.0f, s3)) * fminf(fminf(fabsf(s1), fabsf(s3)), fabsf(0.5f * avg));
  } else if (onesided && xxc > 0.0f) {
    const float d = (fmaf(3.0f, ssc, fmaf(-4.0f, ssup, ss3)) * hh) / xxc;
    const float sg = copysignf(1.0f, s1);
    dsdtau = sg * fmaxf(0.0f, fminf(sg * d, 2.0f * fabsf(s1)));
  }
  herm2_weights(K, dt, rdt, ex, U0, U1, q, xxc, ssup, ssc, dsdtau, Inuup, Inu, plam);
}

static void herm2_first(const or_herm2_c *K, float xxup, float xxc, float xxdn, float ssup, float ssc, float Inuup,
                        float pec, float rpec, float rpedn, float gpc, float *Inu, float *plam)
{
  const float t1 = (xxc - xxup) * K->rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpc = xxc * rpec;
  float mc = fmaf(rxpc, gpc, (pec * fmaf(xxdn, rpedn, -rxpc)) * K->rdsup);
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 3.0f * fabsf(t1)));
  const double dt = herm2_clamp((double)fmaf(K->dsup1, xxup + xxc, K->dsup2 * (t1 - mc)), K->dtmax);
  const double rdt = 1.0 / dt;
  float ex, U0, U1, q;
  pm32((float)dt, &ex, &U0, &U1, &q);
  const float dsdtau = (ssc - ssup) * (float)rdt;
  herm2_weights(K, dt, rdt, ex, U0, U1, q, xxc, ssup, ssc, dsdtau, Inuup, Inu, plam);
}

/* work (nf, nx, ny, 0:nz+1, 3) with the upstream ghost plane set; pe, dpe_dz
 * (nx, ny, nz); g_pe, g_dpe_dz (nx, ny) the ghost's Pe (ghost 1 or 2) or NULL. */
int or_long_char_hermite2(const or_slab_t *s, float *work, float *psi, const float *pe, const float *dpe_dz,
                          const float *g_pe, const float *g_dpe_dz, int ghost, double code_length)
{
  const int nf = s->nf, nx = s->nx, ny = s->ny, nz = s->nz, dir = s->dir;
  if (nz < 2 || ghost < 0 || ghost > 2 || (ghost && (!g_pe || !g_dpe_dz))) return 1;
  const float ds = (float)(s->ds[2]);
  const float dsup = (float)((double)ds / fabs(s->vec[2]));
  or_herm2_c K;
  K.rdsup = 1.0f / dsup;
  K.dsup1 = 0.5f * dsup;
  K.dsup2 = (0.0833333358f * dsup) * dsup;
  K.dtmax = -s->maser_dtau_max;
  K.Imax = (float)s->maser_Inu_max;
  K.get_rates = s->get_psi;
  const float gfac = (float)((double)dir * fabs(s->vec[2]) / code_length);
  const int zs = dir > 0 ? 1 : nz, ze = dir > 0 ? nz : 1;
#define HW(f, x, y, z, k) ((size_t)(f) + (size_t)nf * ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * ((size_t)(z) + (size_t)(nz + 2) * (size_t)(k)))))
#define HP(f, x, y, z) ((size_t)(f) + (size_t)nf * ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * (size_t)((z) - 1))))
#define HC(x, y, z) ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * (size_t)((z) - 1)))
  for (int z = zs; dir > 0 ? z <= ze : z >= ze; z += dir) {
    const int zup = z - dir;
    const int first = z == zs, last = z == ze;
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        const size_t cxy = x + (size_t)nx * y;
        const float pec = pe[HC(x, y, z)], rpec = 1.0f / pec;
        const float gpc = gfac * dpe_dz[HC(x, y, z)];
        float peu = 0.0f, rpeu = 0.0f, gpu = 0.0f;
        if (first && ghost) {
          peu = g_pe[cxy];
          rpeu = 1.0f / peu;
          gpu = gfac * g_dpe_dz[cxy];
        } else if (!first) {
          peu = pe[HC(x, y, zup)];
          rpeu = 1.0f / peu;
          gpu = gfac * dpe_dz[HC(x, y, zup)];
        }
        /* the third parabola sample: downwind, or on the last plane two planes up */
        const int z3 = last ? z - 2 * dir : z + dir;
        float pe3 = 0.0f, rpe3, gp3 = 0.0f;
        if (!last) {
          pe3 = pe[HC(x, y, z3)];
          rpe3 = 1.0f / pe3;
          gp3 = gfac * dpe_dz[HC(x, y, z3)];
        } else if (nz >= 3) {
          rpe3 = 1.0f / pe[HC(x, y, z3)];
        } else {
          rpe3 = ghost == 1 ? 1.0f / g_pe[cxy] : rpec;
        }
        for (int f = 0; f < nf; f++) {
          float I, pl;
          if (first && !ghost)
            herm2_first(&K, work[HW(f, x, y, zup, 0)], work[HW(f, x, y, z, 0)], work[HW(f, x, y, z3, 0)],
                        work[HW(f, x, y, zup, 1)], work[HW(f, x, y, z, 1)], work[HW(f, x, y, zup, 2)], pec, rpec,
                        rpe3, gpc, &I, &pl);
          else
            herm2_step(&K, work[HW(f, x, y, zup, 0)], work[HW(f, x, y, z, 0)], work[HW(f, x, y, z3, 0)],
                       work[HW(f, x, y, zup, 1)], work[HW(f, x, y, z, 1)], work[HW(f, x, y, z3, 1)],
                       work[HW(f, x, y, zup, 2)], peu, rpeu, gpu, pec, rpec, gpc, pe3, rpe3, gp3, !last,
                       last && nz >= 3, &I, &pl);
          work[HW(f, x, y, z, 2)] = I;
          if (psi && K.get_rates) psi[HP(f, x, y, z)] = pl;
        }
      }
  }
#undef HW
#undef HP
#undef HC
  return 0;
}

/* =========================================================================
 * short_char_hermite (rt_solvers_mod.f90:1917-2248), fp32 with the reference's
 * real(8) dtau, 1/dtau and weights: short_char's 4x4 upwind interpolation and
 * 2x2 minimum limiter, applied also to the ratios chi/Pe and Snu/Bnu formed at
 * the upwind grid points (:2014-2026), and the quadratic weights with the
 * product-rule slopes at the target: dchi/ds = (chi/Pe) dPe/ds + Pe d(chi/Pe)/ds
 * with the directional derivative v.grad, clamped to 2 |secant|; dS/dtau =
 * S (dBnu/dtau)/Bnu + Bnu d(S/Bnu)/dtau with the positivity clamp resolved by
 * branch (:2125-2139) so the Lambda diagonal B + C kf (:2155) follows the branch.
 * The first plane takes short_char's linear step.  Periodic x/y; the AMR
 * boundary stencil is not supported.
 * ========================================================================= */
int or_short_char_hermite(const or_slab_t *s, float *work, float *psi, float *irem, float *esc,
                          const float *beta, const float *pe, const float *dpe_dx, const float *dpe_dy,
                          const float *dpe_dz, const float *dlnt_dx, const float *dlnt_dy, const float *dlnt_dz,
                          const float *temp, const float *hknu, double code_length)
{
  const int nf = s->nf, nx = s->nx, ny = s->ny, nz = s->nz, dir = s->dir;
  double xk[4], yk[4], dsup;
  int upo1, upo2;
  or_set_stencil(s->ds, s->vec, xk, yk, &upo1, &upo2, &dsup);
  float kx[4], ky[4];
  for (int i = 0; i < 4; i++) { kx[i] = (float)xk[i]; ky[i] = (float)yk[i]; }
  const double sg = copysign(1.0, s->vec[2]) * (double)dir;
  const float v1 = (float)(s->vec[0] * sg / code_length);
  const float v2 = (float)(s->vec[1] * sg / code_length);
  const float v3 = (float)(s->vec[2] * sg / code_length);
  const float dsup05 = 0.5f * (float)dsup;
  const float rpath = 0.5f / dsup05, dsc2 = (dsup05 * dsup05) / 3.0f;
  const float dtmaxf = -(float)s->maser_dtau_max, Imax = (float)s->maser_Inu_max;
  const double dtmax = -s->maser_dtau_max;
  int *xt = (int *)malloc(sizeof(int) * 4 * nx), *yt = (int *)malloc(sizeof(int) * 4 * ny);
  up_tables_f32(nx, upo1, xt);
  up_tables_f32(ny, upo2, yt);
#define HW(f, x, y, z, k) ((size_t)(f) + (size_t)nf * ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * ((size_t)(z) + (size_t)(nz + 2) * (size_t)(k)))))
#define HP(f, x, y, z) ((size_t)(f) + (size_t)nf * ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * (size_t)((z) - 1))))
#define HC(x, y, z) ((size_t)(x) + (size_t)nx * ((size_t)(y) + (size_t)ny * (size_t)((z) - 1)))
  const int zs = dir > 0 ? 1 : nz, ze = dir > 0 ? nz : 1;
  for (int z = zs; dir > 0 ? z <= ze : z >= ze; z += dir) {
    const int zup = z - dir;
    const int chain = z != zs;
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        float gpe = 0.0f, aT = 0.0f, pec = 0.0f, rpec = 0.0f;
        if (chain) {
          const size_t c = HC(x, y, z);
          gpe = fmaf(v3, dpe_dz[c], fmaf(v2, dpe_dy[c], v1 * dpe_dx[c]));
          aT = fmaf(v3, dlnt_dz[c], fmaf(v2, dlnt_dy[c], v1 * dlnt_dx[c])) / temp[c];
          pec = pe[c];
          rpec = 1.0f / pec;
        }
        for (int f = 0; f < nf; f++) {
          /* the upwind values: fields chi, Snu, Inu and, past the first plane, the ratios */
          const int nfld = chain ? 5 : 3;
          float up[5], mn[5];
          for (int i = 0; i < 5; i++) { up[i] = 0.0f; mn[i] = FLT_MAX; }
          for (int jj = 0; jj < 4; jj++) {
            const int yu = yt[4 * y + jj];
            float row[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            for (int ii = 0; ii < 4; ii++) {
              const int xu = xt[4 * x + ii];
              float v[5];
              v[0] = work[HW(f, xu, yu, zup, 0)];
              v[1] = work[HW(f, xu, yu, zup, 1)];
              v[2] = work[HW(f, xu, yu, zup, 2)];
              if (chain) {
                const float rpe = 1.0f / pe[HC(xu, yu, zup)];
                const float bet = beta[HP(f, xu, yu, zup)];
                v[3] = v[0] * rpe;
                v[4] = (v[1] * (1.0f - bet)) / bet;
              }
              for (int i = 0; i < nfld; i++) {
                row[i] = fmaf(kx[ii], v[i], row[i]);
                if (jj >= 1 && jj <= 2 && ii >= 1 && ii <= 2) mn[i] = fminf(mn[i], v[i]);
              }
            }
            for (int i = 0; i < nfld; i++) up[i] = fmaf(ky[jj], row[i], up[i]);
          }
          for (int i = 0; i < nfld; i++) up[i] = fmaxf(up[i], mn[i]);
          const float xxup = up[0], ssup = up[1], Inuup = up[2];
          const float xx = work[HW(f, x, y, z, 0)], ss = work[HW(f, x, y, z, 1)];
          const size_t p = HP(f, x, y, z);
          if (!chain) {
            float dt = fmaxf(dsup05 * (xxup + xx), dtmaxf);
            float E, W, Psi, Esc;
            lw32(dt, &E, &W, &Psi, &Esc);
            float Inu = fmaf(Psi, ss, fmaf(W, ssup, Inuup * E));
            if (s->split_rates) {
              const int off = dt <= 0 || xx <= 0 || fabsf(Inu) > Imax;
              const float Irem = fmaf(W, ssup, Inuup * E);
              Inu = fmaxf(-Imax, fminf(Imax, Inu));
              Psi = off ? 0.0f : Psi;
              irem[p] = off ? Inu : Irem;
              esc[p] = off ? 1.0f : Esc;
            } else {
              Inu = fmaxf(-Imax, fminf(Imax, Inu));
            }
            work[HW(f, x, y, z, 2)] = Inu;
            if (s->get_psi) psi[p] = (dt > 0 && xx > 0) ? Psi / xx : 0.0f;
            continue;
          }
          const float rxpup = up[3], rhou = up[4];
          const float betc = beta[p];
          const float t1 = (xx - xxup) * rpath;
          const float sgn = copysignf(1.0f, t1);
          const float rxpc = xx * rpec;
          float mc = fmaf(rxpc, gpe, (pec * (rxpc - rxpup)) * rpath);
          mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 2.0f * fabsf(t1)));
          double dt = (double)fmaf(dsup05, xxup + xx, dsc2 * (t1 - mc));
          dt = fmax(copysign(fmax(fabs(dt), (double)1e-20f), dt), dtmax);
          const double rdt = 1.0 / dt;
          const float rdt4 = (float)rdt;
          float ex, U0, U1, q;
          pm32((float)dt, &ex, &U0, &U1, &q);
          const float r1mbc = 1.0f / (1.0f - betc);
          const float Bc = betc * r1mbc;
          const float gc = ((hknu[f] * r1mbc) * aT) / xx;
          const float rhoc = ss / Bc;
          const float t1s = (ss - ssup) * rdt4;
          const float sgns = copysignf(1.0f, t1s);
          float dsdtau = fmaf(ss, gc, (Bc * (rhoc - rhou)) * rdt4);
          float kf, srem;
          if (sgns * dsdtau <= 0.0f) {
            dsdtau = 0.0f;
            kf = 0.0f;
            srem = 0.0f;
          } else if (sgns * dsdtau >= 2.0f * fabsf(t1s)) {
            dsdtau = 2.0f * t1s;
            kf = 2.0f * rdt4;
            srem = -((2.0f * rdt4) * ssup);
          } else {
            kf = gc + rdt4;
            srem = -((Bc * rhou) * rdt4);
          }
          const double B = (2.0 * (double)U1 - (double)q) * rdt;
          const double A = (double)U0 - B;
          const float C = q - U1;
          float Inu = fmaf(C, dsdtau, fmaf((float)B, ss, fmaf((float)A, ssup, Inuup * ex)));
          Inu = fmaxf(-Imax, fminf(Imax, Inu));
          work[HW(f, x, y, z, 2)] = Inu;
          if (s->get_psi) {
            const double pl = B + (double)C * (double)kf;
            const float Psi_loc = (float)pl;
            float ps, rm, es;
            if (dt > 0 && xx > 0 && Psi_loc >= 0.0f && Psi_loc <= 1.0f && fabsf(Inu) < Imax) {
              ps = Psi_loc / xx;
              rm = fmaf(C, srem, fmaf((float)A, ssup, Inuup * ex));
              es = (float)(1.0 - pl);
            } else {
              ps = 0.0f;
              rm = Inu;
              es = 1.0f;
            }
            psi[p] = ps;
            if (s->split_rates) {
              irem[p] = rm;
              esc[p] = es;
            }
          }
        }
      }
  }
#undef HW
#undef HP
#undef HC
  free(xt);
  free(yt);
  return 0;
}

/*
 * or_optab.c -- CPU restatement of the sampled opacity tables of
 * HOP/optab_mod.f90 and the helpers they call (interpol_mod.f90 hermite_coefs,
 * pchip_slopes4/8, pchip_mono4 at the nodes; op_math_mod.f90 searchsorted).
 * TEST INFRASTRUCTURE ONLY.
 *
 * Arithmetic follows the reference's declared kinds: the wavelength slopes and
 * every (ln T, ln ne) -> PC-coordinate step in fp64, the collapse in fp32.  The
 * a*b + c*d sums of the collapse are fused as listed (fmaf), the rest unfused.
 */
#include "or_optab.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>

#define TI(k, it, je) ((size_t)(k) + (size_t)nnu * ((size_t)(it) + (size_t)ntemp * (size_t)(je)))

/* pchip_slopes8 (interpol_mod.f90:240-284) on one line, imin = 1, imax = n */
static void pchip8_line(int n, const double *x, const float *y, size_t ys, float *out, size_t os)
{
#define Y(i) ((double)y[(size_t)(i) * ys])
  const double dx0 = x[1] - x[0], dy0 = Y(1) - Y(0);
  if (n == 2) {
    double a = dy0 / dx0, b = a;
    a = 2.0 * dy0 / dx0 - b;
    b = 2.0 * dy0 / dx0 - a;
    out[0] = (float)a;
    out[os] = (float)b;
    return;
  }
  double prev = 0.0, last = 0.0;   /* slopes of nodes 1 and n-2 (0-based), for the end nodes */
  for (int i = 1; i <= n - 2; i++) {
    const double dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
    const double dym = Y(i) - Y(i - 1), dyp = Y(i + 1) - Y(i);
    double d = 0.0;
    if (!(dym == 0 || dyp == 0)) {
      const double d1 = dym / dxm, d2 = dyp / dxp;
      if (copysign(1.0, d1) == copysign(1.0, d2)) {
        const double alpha = (1.0 + dxm / (dxp + dxm)) / 3.0;
        d = 1.0 / ((1.0 - alpha) / d1 + alpha / d2);
      }
    }
    if (i == 1) prev = d;
    last = d;
    out[(size_t)i * os] = (float)d;
  }
  out[0] = (float)(2.0 * dy0 / dx0 - prev);
  const double dxl = x[n - 1] - x[n - 2], dyl = Y(n - 1) - Y(n - 2);
  out[(size_t)(n - 1) * os] = (float)(2.0 * dyl / dxl - last);
#undef Y
}

/* pchip_slopes4 (interpol_mod.f90:193-235) on one line, imin = 1, imax = n; the
 * node slopes pchip_mono4 returns at the nodes themselves (:335-362) */
static void pchip4_line(int n, const float *x, const float *y, size_t ys, float *out, size_t os)
{
#define Y(i) (y[(size_t)(i) * ys])
  const float dx0 = x[1] - x[0], dy0 = Y(1) - Y(0);
  if (n == 2) {
    float a = dy0 / dx0, b = a;
    a = 2.0f * dy0 / dx0 - b;
    b = 2.0f * dy0 / dx0 - a;
    out[0] = a;
    out[os] = b;
    return;
  }
  float first = 0.0f, last = 0.0f;
  for (int i = 1; i <= n - 2; i++) {
    const float dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
    const float dym = Y(i) - Y(i - 1), dyp = Y(i + 1) - Y(i);
    float d = 0.0f;
    if (!(dym == 0 || dyp == 0)) {
      const double d1 = (double)(dym / dxm), d2 = (double)(dyp / dxp);
      if (copysign(1.0, d1) == copysign(1.0, d2)) {
        const double alpha = (double)((1.0f + dxm / (dxp + dxm)) / 3.0f);
        d = (float)(1.0 / ((1.0 - alpha) / d1 + alpha / d2));
      }
    }
    if (i == 1) first = d;
    last = d;
    out[(size_t)i * os] = d;
  }
  out[0] = 2.0f * dy0 / dx0 - first;
  const float dxl = x[n - 1] - x[n - 2], dyl = Y(n - 1) - Y(n - 2);
  out[(size_t)(n - 1) * os] = 2.0f * dyl / dxl - last;
#undef Y
}

void or_optab_slopes(int nnu, int ntemp, int nne, const double *lam, const float *val, const or_pca_t *pca,
                     float *dl, float *dt, float *de)
{
  float *taxis = (float *)malloc(sizeof(float) * (size_t)ntemp), *eaxis = (float *)malloc(sizeof(float) * (size_t)nne);
  for (int i = 0; i < ntemp; i++) taxis[i] = (float)(pca->c0[0] + (double)i * pca->dc[0]);
  for (int i = 0; i < nne; i++) eaxis[i] = (float)(pca->c0[1] + (double)i * pca->dc[1]);
  for (int je = 0; je < nne; je++)
    for (int it = 0; it < ntemp; it++) pchip8_line(nnu, lam, val + TI(0, it, je), 1, dl + TI(0, it, je), 1);
  for (int je = 0; je < nne; je++)
    for (int k = 0; k < nnu; k++)
      pchip4_line(ntemp, taxis, val + TI(k, 0, je), (size_t)nnu, dt + TI(k, 0, je), (size_t)nnu);
  for (int it = 0; it < ntemp; it++)
    for (int k = 0; k < nnu; k++)
      pchip4_line(nne, eaxis, val + TI(k, it, 0), (size_t)nnu * ntemp, de + TI(k, it, 0), (size_t)nnu * ntemp);
  free(taxis);
  free(eaxis);
}

/* hermite_coefs (interpol_mod.f90:171-188) */
static void hcoefs(float t, float h, float c[5])
{
  const float t2 = t * t, t3 = t2 * t;
  const float p = 3.0f * t2 - 2.0f * t3;
  c[0] = p;
  c[1] = 1.0f - p;
  c[2] = p;
  c[3] = h * ((t3 - 2.0f * t2) + t);
  c[4] = h * (t3 - t2);
}

/* the searchsorted bracket of optab_mod.f90:214/358: k = min(max(searchsorted, 1),
 * nnu - 1), 1-based, which is the number of nodes below x clamped to [1, nnu - 1];
 * returned 0-based with the interval's Hermite coefficients */
static int lam_bracket(int nnu, const double *lam, double x, float c[5])
{
  int lo = 0, hi = nnu;   /* count of lam[i] < x by bisection */
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (lam[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  int k = lo < 1 ? 1 : (lo > nnu - 1 ? nnu - 1 : lo);
  k -= 1;
  const float hl = (float)(lam[k + 1] - lam[k]);
  const float tl = (float)((x - lam[k]) / (lam[k + 1] - lam[k]));
  hcoefs(tl, hl, c);
  return k;
}

/* the per-cell PC coordinates and Hermite coefficients (optab_mod.f90:225-238) */
static void cell_coefs(const or_pca_t *pca, int ntemp, int nne, double temp, double ne, int *it, int *je, float tc[5],
                       float nc[5])
{
  const double d1 = log(temp) - pca->mu[0];
  const double d2 = log(ne) - pca->mu[1];
  const double p1 = pca->rot[0] * d1 + pca->rot[1] * d2;
  const double p2 = pca->rot[2] * d1 + pca->rot[3] * d2;
  const double ft = (p1 - pca->c0[0]) * (1.0 / pca->dc[0]) + 1.0;
  const double fe = (p2 - pca->c0[1]) * (1.0 / pca->dc[1]) + 1.0;
  const double ift = fmin(fmax(floor(ft), 1.0), (double)(ntemp - 1));
  const double ife = fmin(fmax(floor(fe), 1.0), (double)(nne - 1));
  hcoefs((float)(ft - ift), (float)pca->dc[0], tc);
  hcoefs((float)(fe - ife), (float)pca->dc[1], nc);
  *it = (int)ift - 1;
  *je = (int)ife - 1;
}

/* collapse (optab_mod.f90:251-286): wavelength, then temp, then log ne */
static float collapse(int nnu, int ntemp, const float *val, const float *dl, const float *dt, const float *de, int k,
                      int it, int je, const float w[5], const float tc[5], const float nc[5])
{
  const float pl = w[0], wc0 = w[1], wc1 = w[2], wcm0 = w[3], wcm1 = w[4];
  const float opl = 1.0f - pl;
  float v[4], gt[4], ge[4];
  for (int c = 0; c < 4; c++) {
    const size_t a = TI(k, it + (c & 1), je + (c >> 1)), b = a + 1;
    v[c] = fmaf(wcm1, dl[b], fmaf(wcm0, dl[a], fmaf(wc1, val[b], wc0 * val[a])));
    gt[c] = fmaf(pl, dt[b], opl * dt[a]);
    ge[c] = fmaf(pl, de[b], opl * de[a]);
  }
  const float pt = tc[0], opt = 1.0f - pt;
  const float f0 = fmaf(tc[4], gt[1], fmaf(tc[3], gt[0], fmaf(tc[2], v[1], tc[1] * v[0])));
  const float f1 = fmaf(tc[4], gt[3], fmaf(tc[3], gt[2], fmaf(tc[2], v[3], tc[1] * v[2])));
  const float ge0 = fmaf(pt, ge[1], opt * ge[0]);
  const float ge1 = fmaf(pt, ge[3], opt * ge[2]);
  return fmaf(nc[4], ge1, fmaf(nc[3], ge0, fmaf(nc[2], f1, nc[1] * f0)));
}

int or_optab_sample(int nnu, int ntemp, int nne, const double *lam, const or_pca_t *pca, const float *val,
                    const float *dl, const float *dt, const float *de, const float *sv, const float *sl,
                    const float *st, const float *se, long long ncell, const double *temp, const double *ne,
                    const float *chi500, int nf, const double *lam_q, float *back, float *scat)
{
  if (nnu < 2 || ntemp < 2 || nne < 2) return 1;
  for (long long c = 0; c < ncell; c++) {
    int it, je;
    float tc[5], nc[5];
    cell_coefs(pca, ntemp, nne, temp[c], ne[c], &it, &je, tc, nc);
    for (int f = 0; f < nf; f++) {
      float w[5];
      const int k = lam_bracket(nnu, lam, lam_q[f], w);
      const float kap = collapse(nnu, ntemp, val, dl, dt, de, k, it, je, w, tc, nc);
      const float kas = collapse(nnu, ntemp, sv, sl, st, se, k, it, je, w, tc, nc);
      const size_t o = (size_t)f + (size_t)nf * (size_t)c;
      back[o] = (kap + kas) * chi500[c];
      scat[o] = kas * chi500[c];
    }
  }
  return 0;
}

int or_optab_sample_ll(int nnu, int ntemp, int nne, const double *lam, const or_pca_t *pca, const float *val,
                       const float *dl, const float *dt, const float *de, const float *sv, const float *sl,
                       const float *st, const float *se, long long ncell, const double *temp, const double *ne,
                       const float *chi500, const float *vproj, int nf, const double *lam_q, float *xhat,
                       float *ehat, float *chi_scat)
{
  if (nnu < 2 || ntemp < 2 || nne < 2) return 1;
  const int do_scat = chi_scat && sv;
  for (long long c = 0; c < ncell; c++) {
    int it, je;
    float tc[5], nc[5];
    cell_coefs(pca, ntemp, nne, temp[c], ne[c], &it, &je, tc, nc);
    const double vf = 1.0 + (double)vproj[c];
    for (int f = 0; f < nf; f++) {
      float w[5];
      const int k = lam_bracket(nnu, lam, lam_q[f] * vf, w);
      const size_t o = (size_t)f + (size_t)nf * (size_t)c;
      const float add = collapse(nnu, ntemp, val, dl, dt, de, k, it, je, w, tc, nc) * chi500[c];
      xhat[o] = xhat[o] + add;
      ehat[o] = ehat[o] + add;
      if (do_scat) chi_scat[o] = chi_scat[o] + collapse(nnu, ntemp, sv, sl, st, se, k, it, je, w, tc, nc) * chi500[c];
    }
  }
  return 0;
}

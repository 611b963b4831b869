/*
 * or_continuum.c -- CPU restatement of HOP's continuum opacity of a window (see
 * or_continuum.h for the routines followed).  TEST INFRASTRUCTURE ONLY.
 *
 * Kinds follow the Fortran: the tables, xhat, sigma and the interpolation weights
 * are real(4); the EOS state, the absorption factors, the wavelengths and their
 * cubes real(8).  A default-real literal (2.0898E-26, 8./3., 1026., 0.66520e-24,
 * 500., the Rayleigh coefficients) keeps its single-precision value inside real(8)
 * arithmetic; a real(4) array updated from a real(8) expression is rounded once,
 * where the Fortran assigns it.
 */
#include "or_continuum.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

void or_exp4_f32(int n, const float *x, float *y);

static float exp4_1(float x)
{
  float y;
  or_exp4_f32(1, &x, &y);
  return y;
}

static const double OR_RYD = 13.598434, OR_EE = 1.602189e-12, OR_HH = 6.626176e-27, OR_BK = 1.380662e-16;
static const double OR_CC = 2.99792458e10, OR_EM = 9.109534e-28, OR_EC = 4.80325e-10, OR_PI = 3.14159265359;
static const double OR_RBOHR = 5.29177349e-9;

void or_exp_neg0_f32(int n, const float *t, float *E, float *u0);

/* the fits_in test of load_lam_interp_weights: x in [lam(idx), lam(idx+1)), idx
 * 1-based within 1 .. nnu-1 */
static int fits_in(const or_bf_comp_t *c, int idx, double x)
{
  if (!(idx > 0 && idx < c->nnu)) return 0;
  return x >= c->lam[idx - 1] && x < c->lam[idx];
}

/* bftrans_mod.f90:100-198.  Works in the Fortran's 1-based stencil index j and
 * stores it 0-based. */
int or_bf_weights(const or_bf_comp_t *c, int nlam, const double *lam, int *iw, unsigned char *quad, float *lagrange,
                  int *fs, int *fe)
{
  for (int i = 0; i < nlam; i++) {
    iw[i] = -1;
    quad[i] = 0;
    lagrange[3 * i] = lagrange[3 * i + 1] = lagrange[3 * i + 2] = 0.0f;
  }
  double lmin = lam[0], lmax = lam[0];
  for (int i = 1; i < nlam; i++) {
    if (lam[i] < lmin) lmin = lam[i];
    if (lam[i] > lmax) lmax = lam[i];
  }
  if ((!c->maxex && lmin > c->maxl) || (!c->minex && lmax < c->minl)) return 0;
  int lo = nlam, hi = 1;
  int prev = -1;  /* the previous wavelength's 1-based stencil, -1 where none */
  for (int i = 1; i <= nlam; i++) {
    double x = lam[i - 1];
    const int above = x > c->maxl, below = x < c->minl;
    const int skip = (!c->maxex && above) || (!c->minex && below);
    if (skip) {
      prev = -1;
      continue;
    }
    if (i < lo) lo = i;
    if (i > hi) hi = i;
    int j = -1;
    if (below) j = 0;
    else if (above) j = c->nnu;
    else if (i > 1) {
      if (fits_in(c, prev, x)) j = prev;
      else if (fits_in(c, prev - 1, x)) j = prev - 1;
    }
    if (j < 0) {
      for (j = 1; j <= c->nnu - 1; j++)
        if (fits_in(c, j, x)) break;
    }
    int quadratic = c->kvadl;
    if (j < 1 || j >= c->nnu - 1) quadratic = 0;
    else quadratic = quadratic && !c->ldisk[j - 1];
    const int k = quadratic ? 2 : 1;
    if (j > c->nnu - k) j = c->nnu - k;
    if (j < 1) j = 1;
    const double *xx;
    if (c->loglam) {
      x = log(x);
      xx = c->lnlam + (j - 1);
    } else {
      xx = c->lam + (j - 1);
    }
    if (quadratic) {
      const double d1 = x - xx[0], d2 = x - xx[1], d3 = x - xx[2];
      lagrange[3 * (i - 1)] = (float)(d2 * d3 / ((xx[0] - xx[1]) * (xx[0] - xx[2])));
      lagrange[3 * (i - 1) + 1] = (float)(d1 * d3 / ((xx[1] - xx[0]) * (xx[1] - xx[2])));
      lagrange[3 * (i - 1) + 2] = (float)(d1 * d2 / ((xx[2] - xx[0]) * (xx[2] - xx[1])));
    } else {
      const double dx = 1 / (xx[1] - xx[0]);
      lagrange[3 * (i - 1)] = (float)((xx[1] - x) * dx);
      lagrange[3 * (i - 1) + 1] = (float)((x - xx[0]) * dx);
    }
    iw[i - 1] = j - 1;
    quad[i - 1] = (unsigned char)quadratic;
    prev = j;
  }
  *fs = lo - 1;
  *fe = hi - 1;
  return 1;
}

/* absorption_factor (bftrans_mod.f90:476-531) of one cell, times xkap_scale and
 * capped at the real(4) maximum (interp_xkap's scaled_factor, :446-449) */
static float bf_factor(const or_bf_comp_t *c, const or_cont_cells_t *s, int x)
{
  const double ekt = s->e_kT[x], pe = s->pe[x], dxi = s->dxi[x];
  double fk = DBL_MAX;
  switch (c->kind) {
    case OR_BF_HMINUS: fk = c->n[x]; break;
    case OR_BF_NPE: fk = c->n[x] * pe; break;
    case OR_BF_H: {
      if (c->occupation) break;   /* fakt left at huge(1d0): interp_xkap does not use it */
      int k5 = c->k * c->k;
      k5 = k5 * k5 * c->k;
      const double scalar = (double)(2.0898e-26f / (float)(2 * k5));
      fk = scalar * c->level_n[x];
      break;
    }
    case OR_BF_H_FF:
      fk = exp(-ekt * (c->ion_xion - dxi) - c->part[x]);
      fk = (double)2.0898e-26f / (2 * OR_RYD * ekt) * fk * c->n[x];
      break;
    case OR_BF_PAIR: fk = c->n[x] * c->n2[x]; break;
    case OR_BF_H2PLUS: fk = 1e-40 * c->n[x] * c->n2[x]; break;
    case OR_BF_PEDEP: fk = pe * c->n[x]; break;
    case OR_BF_PEACH: fk = pe * c->n[x]; fk = (1e-40 / OR_EE) * ekt * fk; break;
    case OR_BF_MOLECULAR: fk = c->n[x] * c->awgt / 6.023e23; break;
    case OR_BF_REGULAR:
      fk = c->level_g * exp(-ekt * c->level_xion - c->part[x]);
      fk = fk * c->n[x];
      break;
  }
  const double v = fk * c->xkap_scale;
  return (float)(v < (double)FLT_MAX ? v : (double)FLT_MAX);
}

/* one component's table at the cell's temperature, converted to the form of the
 * wavelength interpolation (interp_xkap :284-385 for the table rows it reads) */
typedef struct { int in_bounds, quadratic, it, i; float w[3], dt; int edge; } tinterp_t;

static tinterp_t t_setup(const or_bf_comp_t *c, double temp, double teta)
{
  tinterp_t r;
  memset(&r, 0, sizeof r);
  double t = temp;
  int inb = 1;
  if (!c->minet) inb = inb && (t > c->mint);
  if (!c->maxet) inb = inb && (t < c->maxt);
  r.in_bounds = inb;
  if (!inb) return r;
  t = c->iteta ? teta : temp;
  const int ntt = c->ntt;
  const double *tt = c->tt;
  int it;
  if (t < tt[0]) {
    it = 1;
    r.edge = 1;
  } else if (t >= tt[ntt - 1]) {
    it = ntt - 1;
    r.edge = 2;
  } else {
    for (it = 1; it <= ntt - 1; it++)
      if (tt[it] > t) break;
    r.quadratic = c->kvadt;
  }
  r.it = it;
  if (r.quadratic) {
    const int i = (it + 2 <= ntt) ? it : it - 1;
    const double *t3 = tt + (i - 1);
    const double dt1 = 1. / ((t3[0] - t3[1]) * (t3[0] - t3[2]));
    const double dt2 = 1. / ((t3[1] - t3[0]) * (t3[1] - t3[2]));
    const double dt3 = 1. / ((t3[2] - t3[0]) * (t3[2] - t3[1]));
    const double d1 = t - t3[0], d2 = t - t3[1], d3 = t - t3[2];
    r.w[0] = (float)(d2 * d3 * dt1);
    r.w[1] = (float)(d1 * d3 * dt2);
    r.w[2] = (float)(d1 * d2 * dt3);
    r.i = i;
  } else {
    const double dtdt1 = 1. / (tt[it] - tt[it - 1]);
    r.dt = (float)((t - tt[it - 1]) * dtdt1);
  }
  return r;
}

/* row j (1-based) of the table at the cell's temperature, in the form of the
 * wavelength interpolation */
static float t_row(const or_bf_comp_t *c, const tinterp_t *r, int j)
{
  const float *tab = c->xkap;
  const int nnu = c->nnu;
  float y;
  if (r->quadratic) {
    const int i = r->i;
    y = tab[(j - 1) + (size_t)nnu * (i - 1)] * r->w[0] + tab[(j - 1) + (size_t)nnu * i] * r->w[1] +
        tab[(j - 1) + (size_t)nnu * (i + 1)] * r->w[2];
  } else {
    const int it = r->it;
    const float a = tab[(j - 1) + (size_t)nnu * (it - 1)], b = tab[(j - 1) + (size_t)nnu * it];
    y = (b - a) * r->dt + a;
    if (r->edge == 1) y = fminf(y, tab[j - 1]);
    else if (r->edge == 2) y = fminf(y, tab[(j - 1) + (size_t)nnu * (c->ntt - 1)]);
  }
  const int do_exp = c->log_table && !c->ilogl, do_log = c->ilogl && !c->log_table;
  if (do_exp) y = exp4_1(y);
  else if (do_log) y = logf(fmaxf(y, FLT_MIN));
  return y;
}

/* calc_x_and_k (level_mod.f90:77-94): the hard-sphere volumes of H and He
 * perturbers and the charged-perturber factor of a state of effective quantum
 * number ns.  x**3 is (x*x)*x as gfortran expands a constant integer power; the
 * literals 1.73, 1.02, 8.3e14 and 5.33333333 are default reals. */
static void calc_x_and_k(double ns, double *x1, double *x2, double *k)
{
  const double ns2 = ns * ns;
  const double rih = ns * sqrt(2.5 * ns2 + 0.5);
  const double t1 = OR_RBOHR * (rih + (double)1.73f), t2 = OR_RBOHR * (rih + (double)1.02f);
  *x1 = t1 * t1 * t1;
  *x2 = t2 * t2 * t2;
  double kk = (double)8.3e14f / (ns2 * ns2);
  if (ns > 3.) kk = kk * (double)5.33333333f * ns / ((ns + 1.0) * (ns + 1.0));
  *k = kk * sqrt(kk);
}

/* wcalc2 (level_mod.f90:149-279) for the cells: ab (nlam) is the level's table
 * interpolated to the window (lam^3 included) for fs..fe, times real(xkap_scale) */
static void wcalc2(const or_bf_comp_t *c, int nlam, const double *lam, const float *ab, int fs, int fe, int ncell,
                   const or_cont_cells_t *s, float *chi)
{
  const int li = c->level_i;
  const double hc_e = OR_HH * OR_CC / OR_EE, h_e = OR_HH / OR_EE;
  const double redcut = hc_e / ((pow((double)li, -2.0) - pow((double)(li + 1), -2.0)) * OR_RYD) * 1e8;
  int i5 = li * li;
  i5 = i5 * i5 * li;
  const float q = 2.0898e-26f / (float)(2 * i5);
  /* per wavelength: 0 none, 1 beyond the series limit, 2 below it */
  int *cls = calloc((size_t)nlam, sizeof(int));
  float *g = calloc((size_t)nlam, sizeof(float)), *x1 = calloc((size_t)nlam, sizeof(float));
  float *x2 = calloc((size_t)nlam, sizeof(float)), *kk = calloc((size_t)nlam, sizeof(float));
  double *kd = calloc((size_t)nlam, sizeof(double));
  for (int f = fs; f <= fe; f++) {
    const double cutfac = lam[f] > redcut ? exp((redcut - lam[f]) * 1e-2) : 1.0;
    if (!(cutfac > 1e-1)) continue;
    g[f] = (float)((double)q * cutfac * (double)ab[f]);
    const double nu = OR_CC / lam[f] * (double)1e8f;
    double ns = 1. - (c->level_xion + h_e * nu) / OR_RYD;
    if (ns > 0) {
      ns = 1.0 / sqrt(ns);
      double x1d, x2d, kkd;
      calc_x_and_k(ns, &x1d, &x2d, &kkd);
      cls[f] = 2;
      x1[f] = (float)x1d;
      x2[f] = (float)x2d;
      kk[f] = (float)kkd;
      kd[f] = kkd;
    } else if (!c->dissolved_only) {
      cls[f] = 1;
    }
  }
  const double pi43 = 4.18879;
  for (int x = 0; x < ncell; x++) {
    const float w = (float)c->level_w[x];
    const float omw = (float)(1.0 - c->level_w[x]);
    const double xd = s->shield[x];
    const float xs = (float)xd;
    const float n = (float)c->level_n[x];
    const float ne1 = (float)s->ne[x];
    const float nh43 = (float)(pi43 * c->n[x]);
    const float nhe43 = (float)(pi43 * s->nHeI[x]);
    float *ch = chi + (size_t)nlam * x;
    for (int f = fs; f <= fe; f++) {
      if (cls[f] == 1) {
        ch[f] = ch[f] + w * n * g[f];
      } else if (cls[f] == 2) {
        const float a = nh43 * x1[f] + nhe43 * x2[f];
        float E, omE;
        or_exp_neg0_f32(1, &a, &E, &omE);
        const float k1 = kk[f];
        const float xk = xs * k1;
        float C = 1.0f, omC = 0.0f;
        if (xd * kd[f] < 1e4) {
          const float frac = 0.1402f * xk * k1 / (ne1 * (1.0f + 0.1285f * xk));
          C = frac / (1.0f + frac);
          omC = 1.0f / (1.0f + frac);
        }
        const float d = w > 0.5f ? (omE + E * omC) - omw : w - E * C;
        ch[f] = ch[f] + d * n * g[f];
      }
    }
  }
  free(cls);
  free(g);
  free(x1);
  free(x2);
  free(kk);
  free(kd);
}

/* add_absorption of one component to chi (nlam, ncell) */
static void bf_add(const or_bf_comp_t *c, int nlam, const double *lam, int ncell, const or_cont_cells_t *s, float *chi)
{
  int *iw = malloc(sizeof(int) * nlam);
  unsigned char *quad = malloc((size_t)nlam);
  float *lag = malloc(sizeof(float) * 3 * nlam);
  int fs = 0, fe = -1;
  if (or_bf_weights(c, nlam, lam, iw, quad, lag, &fs, &fe) && c->ntt == 1 && c->kind == OR_BF_H && c->occupation) {
    /* interp_xkap_2 with H_occupation_probability: the table at the window, then
     * wcalc2 for every cell (bftrans_mod.f90:398-428) */
    float *ab = calloc((size_t)nlam, sizeof(float));
    for (int f = fs; f <= fe; f++) {
      float v = 0.0f;
      if (iw[f] >= 0) {
        const float *yy = c->xkap + iw[f];
        v = 0.0f + yy[0] * lag[3 * f];
        v = v + yy[1] * lag[3 * f + 1];
        if (quad[f]) v = v + yy[2] * lag[3 * f + 2];
        if (c->ilogl) v = expf(v);
      }
      if (c->lam3) v = v * (float)(lam[f] * lam[f] * lam[f]);
      ab[f] = v * (float)c->xkap_scale;
    }
    wcalc2(c, nlam, lam, ab, fs, fe, ncell, s, chi);
    free(ab);
  } else if (fe >= fs) {
    for (int x = 0; x < ncell; x++) {
      float *ch = chi + (size_t)nlam * x;
      if (c->ntt > 1) {
        const tinterp_t r = t_setup(c, s->temp[x], s->teta[x]);
        if (!r.in_bounds) continue;
        const float fakt1 = bf_factor(c, s, x);
        for (int f = fs; f <= fe; f++) {
          float ab;
          if (iw[f] >= 0) {
            const int i = iw[f] + 1;
            const float y1 = t_row(c, &r, i), y2 = t_row(c, &r, i + 1);
            const float y3 = t_row(c, &r, i + 2 < c->nnu ? i + 2 : c->nnu);
            ab = y1 * lag[3 * f] + y2 * lag[3 * f + 1] + y3 * lag[3 * f + 2];
          } else {
            ab = c->ilogl ? -FLT_MAX : 0.0f;
          }
          if (c->ilogl) ab = exp4_1(ab);
          if (c->lam3) ab = ab * (float)(lam[f] * lam[f] * lam[f]);
          ch[f] = ch[f] + fakt1 * ab;
        }
      } else {
        const float fakt1 = bf_factor(c, s, x);
        for (int f = fs; f <= fe; f++) {
          float ab;
          if (iw[f] < 0) {
            ab = 0.0f;
          } else {
            const float *yy = c->xkap + iw[f];
            ab = 0.0f + yy[0] * lag[3 * f];
            ab = ab + yy[1] * lag[3 * f + 1];
            if (quad[f]) ab = ab + yy[2] * lag[3 * f + 2];
            if (c->ilogl) ab = expf(ab);
          }
          if (c->lam3) ab = ab * (float)(lam[f] * lam[f] * lam[f]);
          ch[f] = ch[f] + ab * fakt1;
        }
      }
    }
  }
  free(iw);
  free(quad);
  free(lag);
}

int or_continuum_opacities(int ncomp, const or_bf_comp_t *comps, int nlam, const double *lam, const double *nu,
                           int ncell, const or_cont_cells_t *s, const float *beta, float *xhat, float *sigma)
{
  for (int j = 0; j < ncomp; j++)
    if (comps[j].kind < OR_BF_HMINUS || comps[j].kind > OR_BF_REGULAR) return -1;
  const size_t n = (size_t)nlam * ncell;
  memset(xhat, 0, sizeof(float) * n);
  /* add_hrest: the H I levels above n = 15 */
  if (s->nHI) {
    const double nniv2 = (double)(15.5f * 15.5f);
    for (int x = 0; x < ncell; x++) {
      const double ekt = s->e_kT[x], dxi = s->dxi[x];
      double fakt = exp(-ekt * (s->HI_xion - dxi) - s->partHI[x]);
      fakt = (double)2.0898e-26f / (2 * OR_RYD * ekt) * fakt * s->nHI[x];
      if (OR_RYD >= nniv2 * dxi) {
        double hrest = exp(ekt * (OR_RYD / nniv2 - dxi));
        hrest = fakt * (hrest - 1);
        for (int f = 0; f < nlam; f++)
          xhat[(size_t)nlam * x + f] = (float)((double)xhat[(size_t)nlam * x + f] + hrest * (lam[f] * lam[f] * lam[f]));
      }
    }
  }
  int any_istim = 0;
  for (int j = 0; j < ncomp; j++) {
    if (comps[j].istim) any_istim = 1;
    else bf_add(&comps[j], nlam, lam, ncell, s, xhat);
  }
  if (any_istim) {
    float *tmp = calloc(n, sizeof(float));
    float *bet = NULL;
    if (!beta) {
      bet = malloc(sizeof(float) * n);
      for (int x = 0; x < ncell; x++) {
        const double hk_T = (OR_HH / OR_BK) / s->temp[x];
        for (int f = 0; f < nlam; f++) {
          const float b = (float)exp(-nu[f] * hk_T);
          bet[(size_t)nlam * x + f] = b > FLT_MIN ? b : FLT_MIN;
        }
      }
      beta = bet;
    }
    for (int j = 0; j < ncomp; j++)
      if (comps[j].istim) bf_add(&comps[j], nlam, lam, ncell, s, tmp);
    for (size_t k = 0; k < n; k++) xhat[k] = xhat[k] + tmp[k] / (1 - beta[k]);
    free(tmp);
    free(bet);
  }
  if (sigma) {
    memset(sigma, 0, sizeof(float) * n);
    /* thomson = 8./3.*PI*(EC**2/(EM*CC**2))**2, a real(8) parameter */
    const double r = (OR_EC * OR_EC) / (OR_EM * (OR_CC * OR_CC));
    const double thomson = (double)(8.0f / 3.0f) * OR_PI * (r * r);
    for (int x = 0; x < ncell; x++) {
      const double els = thomson * s->ne[x];
      for (int f = 0; f < nlam; f++)
        sigma[(size_t)nlam * x + f] = (float)((double)sigma[(size_t)nlam * x + f] + els);
    }
    for (int x = 0; x < ncell; x++) {
      const double nHI = s->nHI ? s->nHI[x] : 0.0, nHE = s->nHeI ? s->nHeI[x] : 0.0, nH2 = s->nH2 ? s->nH2[x] : 0.0;
      for (int f = 0; f < nlam; f++) {
        double xr = 0.0;
        if (lam[f] > 1400.0) {
          const double m = lam[f] > 1026.0 ? lam[f] : 1026.0;
          xr = 1 / (m * m);
        }
        float *sg = sigma + (size_t)nlam * x + f;
        if (xr > 0.) {
          const double rayh = ((double)5.799e-13f + xr * ((double)1.422e-6f + xr * (double)2.784f)) * nHI;
          const double rayh2 = ((double)8.14e-13f + xr * ((double)1.28e-6f + xr * (double)1.61f)) * nH2;
          *sg = (float)((double)*sg + (rayh + rayh2) * xr * xr);
        }
        double he = 0.0;
        if (s->helium_scattering) {
          const double q = (double)500.f / lam[f];
          const double q2 = q * q;
          he = (double)(0.66520e-24f * 4.f) * (q2 * q2);
        }
        *sg = (float)((double)*sg + he * nHE);
      }
    }
  }
  return 0;
}

/* init_H_levels with compute_shield (composition_mod.f90:2604-2613, 2708-2768) and
 * wcalc (level_mod.f90:108-142), cell by cell as the reference's array statements
 * evaluate them: the shielding, the hydrogenic levels' g exp(-e_kT xion) with xion =
 * RYD (1. - 1./i**2) (a default-real bracket), the occupation probabilities and the
 * partition function 1/sum w n, or exp(-ln U) with the levels above sqrt(RYD/dxi)
 * dissolved when the first cell's dxi > 0; a cell with dxi <= 0 keeps every level
 * (int(sqrt(RYD/0)) has no defined value in the reference). */
void or_h_levels(int ncell, int nk, int occupation, const double *temp, const double *e_kT, const double *ne,
                 const double *dxi, const double *nHI, const double *nHeI, const double *partHI, double *shield,
                 double *level_n, double *level_w)
{
  const double pi43 = 4.18879;
  const int dissolve = !occupation && dxi[0] > 0.0;
  for (int c = 0; c < ncell; c++) {
    double sh = (double)0.08989f * pow(ne[c], 0.16667) / sqrt(temp[c]);
    sh = pow(1.0 + sh, 3.15) / ne[c];
    shield[c] = sh;
  }
  for (int i = 1; i <= nk; i++) {
    const float xi = 1.0f - 1.0f / (float)(i * i);
    const double xion = OR_RYD * (double)xi, g = (double)(2 * i * i);
    for (int c = 0; c < ncell; c++) level_n[c + (size_t)ncell * (i - 1)] = g * exp(-e_kT[c] * xion);
  }
  for (int c = 0; c < ncell; c++) {
    double part;
    if (occupation) {
      part = 0.0;
      for (int i = 1; i <= nk; i++) {
        double x1, x2, k1;
        calc_x_and_k((double)i, &x1, &x2, &k1);
        const double k2 = k1 * k1;
        const double x = shield[c];
        double res = exp(-(pi43 * (nHI[c] * x1 + nHeI[c] * x2)));
        if (k1 * x < 1e4) {
          const double frac = 0.1402 * x * k2 / (ne[c] * (1.0 + (double)0.1285f * x * k1));
          res = res * (frac / (1.0 + frac));
        }
        level_w[c + (size_t)ncell * (i - 1)] = res;
        part = part + res * level_n[c + (size_t)ncell * (i - 1)];
      }
      part = 1.0 / part;
    } else {
      part = exp(-partHI[c]);
      if (dissolve && dxi[c] > 0.0) {
        const double h1 = sqrt(OR_RYD / dxi[c]);
        const int nniv = h1 < 2147483647.0 ? (int)h1 : 2147483647;
        for (int i = 1; i <= nk; i++) {
          double *n = &level_n[c + (size_t)ncell * (i - 1)];
          if (nniv < i) *n = 0.0;
          else if (nniv == i) *n = *n * (h1 - (double)nniv);
        }
      }
    }
    for (int i = 1; i <= nk; i++) {
      double *n = &level_n[c + (size_t)ncell * (i - 1)];
      *n = nHI[c] * *n * part;
    }
  }
}

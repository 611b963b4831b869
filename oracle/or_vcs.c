/*
 * or_vcs.c -- CPU restatement of the tabulated hydrogen profiles of
 * HOP/hvcs_mod.f90 (VCS tables of Lemke 1997 or Stehle & Hutcheon 1999):
 * read_vcs_grid, vcs_row/vcs_supported/vcs_resonance/vcs_radiative,
 * vcs_prepare with vcs_cell_profile, qpol, qpol_w, qpol4, bracket, tail_coef,
 * vcs_eval and vcs_tail.  TEST INFRASTRUCTURE ONLY.
 *
 * Kinds as declared there: the grid, its axes and the cell profile are float
 * (pchip_slopes4 keeps its harmonic mean in double), the profile evaluation and
 * the tail double.  Nothing is contracted.
 */
#include "or_vcs.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#define NW OR_VCS_NW
#define NH OR_VCS_NH
#define NT OR_VCS_NT
#define NE OR_VCS_NE
#define NL OR_VCS_NL

static or_vcs_series_t g_ser[3];
static int g_loaded = 0;

static const double LN10 = 2.30258509299404568402;
static const double AA_PER_S = 2.99792458e10 * 1.e8;

/* pchip_slopes4 (interpol_mod.f90:193-235): the interior slope of node i (0-based) */
static float pchip4_interior(const float *x, const float *y, int i)
{
  const float dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
  const float dym = y[i] - y[i - 1], dyp = y[i + 1] - y[i];
  if (dym == 0 || dyp == 0) return 0.0f;
  const double d1 = (double)(dym / dxm), d2 = (double)(dyp / dxp);
  if (copysign(1.0, d1) != copysign(1.0, d2)) return 0.0f;
  const double alpha = (double)((1.0f + dxm / (dxp + dxm)) / 3.0f);
  return (float)(1.0 / ((1.0 - alpha) / d1 + alpha / d2));
}

/* pchip_slopes4 over the window imin = j, imax = j + 1 (0-based j, n >= 3 nodes): the
 * two slopes it computes there, the end rules included */
static void pchip4_pair(const float *x, const float *y, int n, int j, float *sj, float *sj1)
{
  if (j == 0) *sj = 2.0f * (y[1] - y[0]) / (x[1] - x[0]) - pchip4_interior(x, y, 1);
  else *sj = pchip4_interior(x, y, j);
  if (j + 1 == n - 1) *sj1 = 2.0f * (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]) - pchip4_interior(x, y, n - 2);
  else *sj1 = pchip4_interior(x, y, j + 1);
}

/* pchip_slopes4 over all nodes (imin = 1, imax = n), for the stored T slopes */
static void pchip4_all(const float *x, const float *y, int n, float *s)
{
  if (n == 2) {
    float a = (y[1] - y[0]) / (x[1] - x[0]), b = a;
    a = 2.0f * (y[1] - y[0]) / (x[1] - x[0]) - b;
    b = 2.0f * (y[1] - y[0]) / (x[1] - x[0]) - a;
    s[0] = a;
    s[1] = b;
    return;
  }
  for (int i = 1; i <= n - 2; i++) s[i] = pchip4_interior(x, y, i);
  s[0] = 2.0f * (y[1] - y[0]) / (x[1] - x[0]) - s[1];
  s[n - 1] = 2.0f * (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]) - s[n - 2];
}

/* hermite_value4 (interpol_mod.f90:125-140) */
static float hermite4(float t, float h, float y0, float y1, float m0, float m1)
{
  const float t2 = t * t, t3 = t2 * t;
  const float p = 3.0f * t2 - 2.0f * t3;
  return (1.0f - p) * y0 + p * y1 + h * (((t3 - 2.0f * t2) + t) * m0 + (t3 - t2) * m1);
}

/* read_vcs_grid (hvcs_mod.f90:145-208) */
int or_vcs_load(int s, const char *fname, int radiative)
{
  if (s < 1 || s > 3) return 1;
  or_vcs_series_t *S = &g_ser[s - 1];
  memset(S, 0, sizeof *S);
  FILE *f = fopen(fname, "r");
  if (!f) return 2;
  float dw0, ddw, ne0, dne, nh0, dnh, lgt0, dlgt;
  if (fscanf(f, "%f %f %f %f %f %f %f %f", &dw0, &ddw, &ne0, &dne, &nh0, &dnh, &lgt0, &dlgt) != 8) {
    fclose(f);
    return 3;
  }
  int k = 0;
  while (k < NL) {
    int lo, up, nn;
    if (fscanf(f, "%d %d %d", &lo, &up, &nn) != 3) break;
    if (nn < 1 || nn > NH) {
      fclose(f);
      return 4;
    }
    int ok = 1;
    for (int l = 0; l < NE && ok; l++)
      for (int kk = 0; kk < NT && ok; kk++)
        for (int j = 0; j < nn && ok; j++)
          for (int i = 0; i < NW && ok; i++)
            ok = fscanf(f, "%f", &S->grid[k][l][kk][j][i]) == 1;
    if (!ok) break;
    S->nlow[k] = lo;
    S->nup[k] = up;
    S->nhhnr[k] = nn;
    k++;
  }
  fclose(f);
  S->nlines = k;
  if (k < 1) return 5;
  for (int i = 0; i < NW; i++) S->nw[i] = dw0 + (float)i * ddw;
  for (int i = 0; i < NT; i++) S->nt[i] = lgt0 + (float)i * dlgt;
  for (int i = 0; i < NE; i++) S->ne[i] = ne0 + (float)i * dne;
  for (int i = 0; i < NH; i++) S->nh[i] = nh0 + (float)i * dnh;
  for (int i = 0; i < NW; i++) S->dw_lin[i] = powf(10.0f, S->nw[i]);
  S->dw_first = pow(10.0, (double)S->nw[0]);
  S->dw_last = pow(10.0, (double)S->nw[NW - 1]);
  S->nw_invdx = 1.0f / ddw;
  for (int kk2 = 0; kk2 < k; kk2++) {
    if (S->nhhnr[kk2] > 1) continue;
    for (int l = 0; l < NE; l++)
      for (int i = 0; i < NW; i++) {
        float col[NT], sl[NT];
        for (int t = 0; t < NT; t++) col[t] = S->grid[kk2][l][t][0][i];
        pchip4_all(S->nt, col, NT, sl);
        for (int t = 0; t < NT; t++) S->tslope[kk2][l][t][i] = sl[t];
      }
  }
  S->radiative = radiative;
  S->loaded = 1;
  g_loaded = 1;
  return 0;
}

void or_vcs_clear(void)
{
  memset(g_ser, 0, sizeof g_ser);
  g_loaded = 0;
}

const or_vcs_series_t *or_vcs_series(int s) { return (s >= 1 && s <= 3 && g_ser[s - 1].loaded) ? &g_ser[s - 1] : 0; }

/* vcs_row (hvcs_mod.f90:243-256), 0-based row or -1 */
int or_vcs_row(int n, int m)
{
  const int s = n - 1;
  if (s < 1 || s > 3 || !g_ser[s - 1].loaded) return -1;
  for (int k = 0; k < g_ser[s - 1].nlines; k++)
    if (g_ser[s - 1].nlow[k] == n && g_ser[s - 1].nup[k] == m) return k;
  return -1;
}

int or_vcs_supported(int n, int m) { return g_loaded && or_vcs_row(n, m) >= 0; }
int or_vcs_resonance(int n, int m) { return g_ser[n - 2].nhhnr[or_vcs_row(n, m)] > 1; }
int or_vcs_radiative(int n) { return g_ser[n - 2].radiative; }

/* qpol (hvcs_mod.f90:431-466) */
static float qpol(float x, const float *a, const float *f, int no)
{
  int k = no - 1;          /* 1-based, as the Fortran */
  if (x > a[no - 1]) goto l50;
  k = 1;
  if (x < a[0] || no == 2) goto l50;
  {
    int nn = no;
    for (;;) {
      if (k == nn - 1) break;
      const int i = (k + nn) / 2;
      if (a[i - 1] >= x) nn = i;
      else k = i;
    }
    if (k == no - 1) k = k - 1;
    const float u = x - a[k - 1], v = x - a[k], w = x - a[k + 1];
    const float y = (f[k - 1] - f[k]) / (v - u);
    const float z = (f[k] - f[k + 1]) / (w - v);
    if (y * z > 0.0f) return f[k - 1] + u * y / (1.0f - v * (y - z) / (f[k - 1] - f[k + 1]));
    return f[k - 1] + u * (y + v * (y - z) / (w - u));
  }
l50:
  return f[k - 1] + (f[k] - f[k - 1]) * (x - a[k - 1]) / (a[k] - a[k - 1]);
}

/* qpol_w (hvcs_mod.f90:472-503) on the wavelength axis of series s */
static float qpol_w(float x, const or_vcs_series_t *S, const float *f)
{
  const float *a = S->nw;
  int k;
  if (x > a[NW - 1]) {
    k = NW - 2;
    return f[k] + (f[k + 1] - f[k]) * (x - a[k]) / (a[k + 1] - a[k]);
  } else if (x < a[0]) {
    k = 0;
    return f[k] + (f[k + 1] - f[k]) * (x - a[k]) / (a[k + 1] - a[k]);
  }
  k = (int)((x - a[0]) * S->nw_invdx) + 1;
  if (k < 1) k = 1;
  if (k > NW - 2) k = NW - 2;
  k -= 1;   /* 0-based */
  const float u = x - a[k], v = x - a[k + 1], w = x - a[k + 2];
  const float y = (f[k] - f[k + 1]) / (v - u);
  const float z = (f[k + 1] - f[k + 2]) / (w - v);
  if (y * z > 0.0f) return f[k] + u * y / (1.0f - v * (y - z) / (f[k] - f[k + 2]));
  return f[k] + u * (y + v * (y - z) / (w - u));
}

/* bracket (hvcs_mod.f90:508-520), 0-based */
static int bracket(float x, const float *a, int n)
{
  int j = 0;
  for (int kk = 0; kk < n - 1; kk++)
    if (x >= a[kk]) j = kk;
  return j;
}

/* qpol4 (hvcs_mod.f90:528-554) */
static float qpol4(float x, const float *a, const float *f, int no)
{
  if (no < 3) return qpol(x, a, f, no);
  const int j = bracket(x, a, no);
  float sj, sj1;
  pchip4_pair(a, f, no, j, &sj, &sj1);
  const float h = a[j + 1] - a[j];
  const float t = (x - a[j]) / h;
  return hermite4(t, h, f[j], f[j + 1], sj, sj1);
}

/* vcs_cell_profile (hvcs_mod.f90:349-426) */
static int vcs_cell_profile(int n, int m, float temp, float ne, float nh, float *lp, float *lognorm)
{
  for (int i = 0; i < NW; i++) lp[i] = 0.0f;
  *lognorm = 0.0f;
  const int r = or_vcs_row(n, m);
  if (r < 0) return 0;
  const or_vcs_series_t *S = &g_ser[n - 2];
  const int nn = S->nhhnr[r];
  float tlog = log10f(fmaxf(temp, 1.0f));
  float nelog = log10f(fmaxf(ne, 1.0f));
  float nhlog = log10f(fmaxf(nh, 1.0f));
  if (nelog < S->ne[0]) nelog = S->ne[0];
  nelog = fminf(nelog, S->ne[NE - 1]);
  tlog = fminf(fmaxf(tlog, S->nt[0]), S->nt[NT - 1]);
  if (nn > 1) nhlog = fminf(fmaxf(nhlog, S->nh[0]), S->nh[nn - 1]);
  const int jt = bracket(tlog, S->nt, NT);
  const float ht = S->nt[jt + 1] - S->nt[jt];
  const float tt = (tlog - S->nt[jt]) / ht;
  const int je = bracket(nelog, S->ne, NE);
  const float he = S->ne[je + 1] - S->ne[je];
  const float te = (nelog - S->ne[je]) / he;
  const int le0 = je - 1 < 0 ? 0 : je - 1;
  const int le1 = je + 2 > NE - 1 ? NE - 1 : je + 2;
  const int ns = le1 - le0 + 1;
  for (int i = 0; i < NW; i++) {
    float ve[NE];
    for (int l = le0; l <= le1; l++) {
      if (nn > 1) {
        float vt[NT];
        for (int kk = 0; kk < NT; kk++) {
          float vh[NH];
          for (int j = 0; j < nn; j++) vh[j] = S->grid[r][l][kk][j][i];
          vt[kk] = qpol4(nhlog, S->nh, vh, nn);
        }
        ve[l] = qpol4(tlog, S->nt, vt, NT);
      } else {
        ve[l] = hermite4(tt, ht, S->grid[r][l][jt][0][i], S->grid[r][l][jt + 1][0][i], S->tslope[r][l][jt][i],
                         S->tslope[r][l][jt + 1][i]);
      }
    }
    float sj, sj1;
    pchip4_pair(S->ne + le0, ve + le0, ns, je - le0, &sj, &sj1);
    lp[i] = hermite4(te, he, ve[je], ve[je + 1], sj, sj1);
  }
  float plin = powf(10.0f, lp[0]);
  float area = plin * S->dw_lin[0];
  for (int i = 0; i < NW - 1; i++) {
    const float dl = S->dw_lin[i + 1] - S->dw_lin[i];
    const float plin_next = powf(10.0f, lp[i + 1]);
    area = area + 0.5f * (plin + plin_next) * dl;
    plin = plin_next;
  }
  area = 2.0f * area;
  *lognorm = log10f(area);
  return 1;
}

/* vcs_prepare + tail_coef (hvcs_mod.f90:262-282, 319-327) */
void or_vcs_prepare(int n, int m, double nu0, float temp, float ne, float nh, or_vcs_cell_t *c)
{
  float lognorm;
  c->ok = vcs_cell_profile(n, m, temp, ne, nh, c->lp, &lognorm);
  c->lognorm = (double)lognorm;
  c->lam0 = AA_PER_S / nu0;
  c->q_tail = g_ser[0].dw_last / c->lam0;
  c->ts = c->ta = 0.0;
  if (c->ok) {
    const double a = (double)g_ser[0].nw[NW - 2];
    const double slope = (double)(c->lp[NW - 1] - c->lp[NW - 2]) / (double)(g_ser[0].nw[NW - 1] - g_ser[0].nw[NW - 2]);
    c->ts = slope;
    c->ta = LN10 * ((double)c->lp[NW - 2] - slope * a - c->lognorm) + (1.0 + slope) * log(c->lam0);
  }
}

/* vcs_eval (hvcs_mod.f90:286-313) */
double or_vcs_eval(const or_vcs_cell_t *c, double q)
{
  if (!c->ok) return 0.0;
  const double dlam = fabs(q) * c->lam0;
  const double deltaw = log10(fmax(dlam, g_ser[0].dw_first));
  const double p = (double)qpol_w((float)deltaw, &g_ser[0], c->lp);
  return exp(LN10 * (p - c->lognorm)) * c->lam0;
}

/* vcs_tail (hvcs_mod.f90:333-343) */
double or_vcs_tail(const or_vcs_cell_t *c, double lnq) { return c->ok ? exp(c->ta + c->ts * lnq) : 0.0; }

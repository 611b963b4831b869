/*
 * or_stateq.c -- CPU restatement of the statistical-equilibrium step of
 * OpenMULTI3D.  TEST INFRASTRUCTURE ONLY (the checker of the SE kernels).
 *
 *   classic_col (electron collisions)   SRC/atom_mod.f90:1758-1850
 *   expin, Kramer, gaunt                SRC/atom_mod.f90:2362-2467
 *   setup_transition_matrix             SRC/atom_mod.f90:740-841
 *   line_rate_coefficients              SRC/atom_mod.f90:862-884
 *   lineq / lineq_no_pivot              HOP/op_math_mod.f90:263-356, 420-449
 *   update_populations (per cell)       SRC/atom_mod.f90:439-732
 *   ng_accumulate / ng_extrapolate      SRC/ng_mod.f90:241-392
 *
 * Fortran constants written without a kind suffix are default (single
 * precision) reals even inside real(8) expressions; they appear below as
 * float literals so that the double arithmetic sees the same numbers
 * (the expin and gaunt tables, 0.2, 0.1, 0.3, 1.55e13, 1e-16, fmin=1e-6).
 * Compiled with -ffp-contract=off: every product and sum is rounded once,
 * in the order the Fortran expression evaluates it.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "or_stateq.h"

/* HOP/const_mod.f90:14-77 */
#define SQ_PI 3.14159265359
#define SQ_EE 1.602189e-12
#define SQ_EM 9.109534e-28
#define SQ_BK 1.380662e-16
#define SQ_HH 6.626176e-27
#define SQ_CC 2.99792458e10
#define SQ_RBOHR 5.29177349e-9
#define SQ_E_K (SQ_EE / SQ_BK)
#define SQ_RYDK (13.605 * SQ_E_K)
#define SQ_RYDV 13.605
#define SQ_HZ_TO_AA (SQ_CC / 1e-8)
#define SQ_AA_TO_HZ (1e-8 / SQ_CC)
#define SQ_H_E (SQ_HH / SQ_EE)
/* kramer_const = 64 PI^4 EC^10 EM / (3 sqrt(3) CC HH^6) (atom_mod.f90:2414) as the
 * compiler folds it: every power and product rounded to double once */
#define SQ_KRAMER_CONST 0x1.c6dc1aa1038f0p+97
#define SQ_MH 1.6726e-24
/* ame is a default-real literal in the reference (atom_mod.f90:220-222) */
#define SQ_AME ((double)5.485799e-4f)
#define SQ_AMH 1.0
#define SQ_MU_E (SQ_AME / (SQ_AME + SQ_AMH))
#define SQ_ERYD (13.605 * SQ_EE)

/* expin: E1(x) by rational approximations, 0 for x <= 0 (atom_mod.f90:2362-2397) */
double sq_expin(double x)
{
  static const float a[6] = {-44178.5471728217f, 57721.7247139444f, 9938.31388962037f,
                             1842.11088668000f, 101.093806161906f, 5.03416184097568f};
  static const float b[5] = {76537.3323337614f, 32597.1881290275f, 6106.10794245759f,
                             635.419418378382f, 37.2298352833327f};
  static const float c[7] = {4.65627107975096e-7f, .999979577051595f, 9.04161556946329f,
                             24.3784088791317f, 23.0192559391333f, 6.90522522784444f, .430967839469389f};
  static const float d[6] = {10.0411643829054f, 32.4264210695138f, 41.2807841891424f,
                             20.4494785013794f, 3.31909213593302f, .103400130404874f};
  static const float e[7] = {-.999999999998447f, -26.6271060431811f, -241.055827097015f,
                             -895.927957772937f, -1298.85688746484f, -545.374158883133f, -5.66575206533869f};
  static const float f[6] = {28.6271060422192f, 292.310039388533f, 1332.78537748257f,
                             2777.61949509163f, 2404.01713225909f, 631.657483280800f};
  const double ex = exp(-x);
  if (x > 4) {
    return (ex + ex * (e[0] + (e[1] + (e[2] + (e[3] + (e[4] + (e[5] + e[6] / x) / x) / x) / x) / x) / x) /
                     (x + f[0] + (f[1] + (f[2] + (f[3] + (f[4] + f[5] / x) / x) / x) / x) / x)) /
           x;
  } else if (x > 1) {
    return ex * (c[6] + (c[5] + (c[4] + (c[3] + (c[2] + (c[1] + c[0] * x) * x) * x) * x) * x) * x) /
           (d[5] + (d[4] + (d[3] + (d[2] + (d[1] + (d[0] + x) * x) * x) * x) * x) * x);
  } else if (x > 0) {
    return (a[0] + (a[1] + (a[2] + (a[3] + (a[4] + a[5] * x) * x) * x) * x) * x) /
               (b[0] + (b[1] + (b[2] + (b[3] + (b[4] + x) * x) * x) * x) * x) -
           log(x);
  }
  return 0.0;
}

/* bound-free Gaunt factor (atom_mod.f90:2436-2467) */
double sq_gaunt(double lam, int n)
{
  static const float a1[6] = {1.078e00f, 1.0926e0f, 1.0983e0f, 1.0954e0f, 1.0912e0f, 1.0925e0f};
  static const float b1[6] = {-8.754e14f, -2.019e14f, -9.45e13f, -5.188e13f, -3.2e13f, -2.331e13f};
  static const float c1[6] = {-1.791e29f, 1.836e28f, 9.177e27f, 3.552e27f, 1.576e27f, 9.325e26f};
  static const float a2[6] = {0.798e00f, 0.768e00f, 0.793e00f, 0.831e00f, 0.758e00f, 0.79e00f};
  static const float b2[6] = {5.358e15f, 6.242e15f, 5.48e15f, 4.094e15f, 6.633e15f, 5.808e15f};
  static const float c2[6] = {-3.484e31f, -3.208e31f, -2.318e31f, -1.43e31f, -3.32e31f, -2.844e31f};
  const double inv_nu = lam * SQ_AA_TO_HZ;
  if (n > 6) return 1.0;
  if (inv_nu >= (double)1e-16f) return a1[n - 1] + (b1[n - 1] + c1[n - 1] * inv_nu) * inv_nu;
  return a2[n - 1] + (b2[n - 1] + c2[n - 1] * inv_nu) * inv_nu;
}

/* Kramers' hydrogenic cross section (atom_mod.f90:2404-2420); nl**5 and nu**3
 * are the multiplication chains of an integer power */
double sq_kramer(double lam, double dev)
{
  const double nu = SQ_HZ_TO_AA / lam;
  if (dev > 0) {
    const double nl = sqrt(SQ_RYDV / dev);
    const double nl2 = nl * nl, nl5 = nl * (nl2 * nl2), nu3 = nu * (nu * nu);
    return SQ_KRAMER_CONST * sq_gaunt(lam, (int)ceil(nl)) / (nl5 * nu3);
  }
  return 0.0;
}

/* prepare_Drawin (atom_mod.f90:1741-1750): 16 pi a0^2 sqrt(2k / (pi m_H A mu_H)) mu_e / mu_H
 * with mu_H = 1 / (A + 1); const is folded at compile time in the reference, each
 * operation rounded to double */
double sq_prepare_drawin(double awgt)
{
  const double c = (16 * SQ_PI) * (SQ_RBOHR * SQ_RBOHR);
  const double mu_h = SQ_AMH / (awgt + SQ_AMH);
  const double drmu = SQ_PI * SQ_MH * awgt * mu_h;
  return c * sqrt(2.0 * SQ_BK / drmu) * SQ_MU_E / mu_h;
}

void sq_hermite_derivative(int n, const double *x, const double *y, double *d)
{
#define DX(i) (x[(i) + 1] - x[(i)])
#define DY(i) (y[(i) + 1] - y[(i)])
  for (int i = 0; i < n; i++) d[i] = 0.0;
  if (n == 2) {
    d[0] = DY(0) / DX(0);
    d[1] = d[0];
  }
  for (int i = 1; i <= n - 2; i++) {
    if (DY(i - 1) == 0 || DY(i) == 0) continue;
    const double d1 = DY(i - 1) / DX(i - 1), d2 = DY(i) / DX(i);
    if (copysign(1.0, d1) == copysign(1.0, d2)) {
      const double alpha = (1.0 + DX(i - 1) / (DX(i) + DX(i - 1))) / 3.0;
      d[i] = 1.0 / ((1.0 - alpha) / d1 + alpha / d2);
    }
  }
  d[0] = 2.0 * DY(0) / DX(0) - d[1];
  d[n - 1] = 2.0 * DY(n - 2) / DX(n - 2) - d[n - 2];
#undef DX
#undef DY
}

/* BinarySearch8 (op_math_mod.f90:179-199), 1-based as there: arr(l) < x <= arr(r) */
static int sq_bsearch8(const double *arr, int l, int r, double x)
{
  if (r - l > 1) {
    const int mid = l + (r - l) / 2;
    if (arr[mid - 1] >= x) return sq_bsearch8(arr, l, mid, x);
    return sq_bsearch8(arr, mid, r, x);
  }
  return l;
}

double sq_hermite_interp(int n, const double *x, const double *y, const double *d, double xx)
{
  if (xx <= x[0]) return y[0];
  if (xx >= x[n - 1]) return y[n - 1];
  const int i = sq_bsearch8(x, 1, n, xx) - 1;
  const double dx = x[i + 1] - x[i];
  /* hermite_value8 (interpol_mod.f90:149-162) */
  const double t = (xx - x[i]) / dx;
  const double t2 = t * t, t3 = t2 * t;
  const double p = 3.0 * t2 - 2.0 * t3;
  return (1.0 - p) * y[i] + p * y[i + 1] + dx * ((t3 - 2.0 * t2 + t) * d[i] + (t3 - t2) * d[i + 1]);
}

/* gencol (atom_mod.f90:2223-2360) for one record and cell: upward and downward rate */
static void sq_gencol_record(const sq_atom_t *at, int r, double temp, double ne, double dxi, double e_kT,
                             double lsaha, double nh1, double n_collider, double nll, double nul, double *cup,
                             double *cdn)
{
  const double c0 = ((SQ_ERYD / sqrt(SQ_EM)) * SQ_PI * (SQ_RBOHR * SQ_RBOHR)) * sqrt(8.0 / (SQ_PI * SQ_BK));
  const int ll = at->gll[r], ul = at->gul[r];
  double u = 0, d = 0, nji;
  double dev = at->ev[ul] - at->ev[ll];
  if (at->ion[ul] > at->ion[ll]) {
    const int ii = at->ion[ll] * (at->ion[ll] - 1), jj = at->ion[ul] * (at->ion[ul] - 1);
    dev = dev - dxi * 0.5 * (jj - ii);
  }
  if (nll > 0) {
    nji = nul / nll;
  } else {
    const double tns = -dev * e_kT + (at->ion[ul] - at->ion[ll]) * lsaha;
    nji = at->g[ul] / at->g[ll] * exp(tns);
  }
  const double stg = sqrt(temp);
  const size_t o = (size_t)r * at->ntemp;
  const double ct = exp(sq_hermite_interp(at->ntemp, at->gt, at->glnc + o, at->gdc + o, temp));
  switch (at->gkind[r]) {
  case SQ_GC_OHM:
    d = c0 / at->g[ul] * ct * ne / stg;
    u = d * nji;
    break;
  case SQ_GC_CE:
    d = at->g[ll] / at->g[ul] * ct * ne * stg;
    d = d * at->cbbesc;
    u = d * nji;
    break;
  case SQ_GC_CH:
    d = ct * nh1;
    d = d * at->cbbhsc;
    u = d * nji;
    break;
  case SQ_GC_CHI:
    u = ct * nh1;
    u = u * at->cbfhsc;
    d = u / nji;
    break;
  case SQ_GC_CI:
    u = ct * ne * stg * exp(-(at->ev[ul] - at->ev[ll]) * e_kT);
    u = u * at->cbfesc;
    d = u / nji;
    break;
  case SQ_GC_CH0:
    u = ct * nh1;
    if (at->ch0_hmip) u = u * exp(-(double)0.754f * e_kT);
    u = u * at->cbfhsc;
    d = u / nji;
    break;
  case SQ_GC_UP:
    u = ct * n_collider;
    d = u / nji;
    break;
  case SQ_GC_DN:
    d = ct * n_collider;
    u = d * nji;
    break;
  default:
    break;
  }
  *cup = u * at->colscale;
  *cdn = d * at->colscale;
}

/* classic_col (atom_mod.f90:1758-1880): cup(cell, pair) [1/s] upward, colscale
 * applied, the electron recipe's rate in rows 0..ncol-1 and, with chkind, the
 * hydrogen recipe's in rows ncol..2ncol-1; the downward rate of each is
 * cup * n*_i/n*_j */
void or_collisions(const sq_atom_t *at, int ncell, const double *temp, const double *ne, const double *e_kT,
                   const double *dxi, const double *nh1, const double *nstar, const double *lsaha,
                   const double *coll, double *cup)
{
  const double sq32 = sqrt(3.0) / 2.0;
  const double sqr3_2pi = sq32 / SQ_PI;
  const double sq8bmp = sqrt(8 * SQ_BK / SQ_EM / SQ_PI);
  const double c0 = SQ_PI * (SQ_RBOHR * SQ_RBOHR) * sq8bmp;
  const int ncol = at->ncol;
  for (int c = 0; c < ncell; c++) {
    const double sqt = sqrt(temp[c]);
    const double allen = c0 * SQ_RYDK * ne[c] / sqt;
    const double regemorter = 14.5 * allen * SQ_RYDK / SQ_E_K;
    const double seaton = (double)1.55e13f * ne[c] / sqt;
    for (int p = 0; p < ncol; p++) {
      const int i = at->ci[p], j = at->cj[p];
      const int cont = at->ion[j] > at->ion[i];
      double fac = at->cfac[p], f = 0;
      double dev = at->ev[j] - at->ev[i];
      dev = fmax(dev, 1e-8);
      if (cont) {
        const int jj = at->ion[j] * (at->ion[j] - 1), ii = at->ion[i] * (at->ion[i] - 1);
        dev = dev - (dxi ? dxi[c] : 0.0) * 0.5 * (jj - ii);
      } else {
        f = fmax(fac, at->fmin * at->g[j]);
      }
      const double u0 = dev * e_kT[c];
      const double ex = exp(-u0);
      double v = 0;
      if (cont && at->ckind[p] == SQ_COL_SEATON) {
        if (fac == 0) {
          const double lam0 = SQ_HZ_TO_AA * SQ_H_E / dev;
          fac = sq_kramer(lam0, dev);
        }
        const double tmp = (double)fminf(0.1f * (float)at->ion[i], 0.3f);
        v = seaton * fac * tmp / u0 * ex;
        v = v * at->cbfesc;
      } else if (!cont && at->ckind[p] == SQ_COL_REGEMORTER) {
        const double tmp = fmax((double)0.2f * ex, sqr3_2pi * sq_expin(u0));
        v = regemorter * f * tmp / dev;
        v = fmax(v, allen * at->upsilon_floor * ex / at->g[i]);
        v = v * at->cbbesc;
      }
      if (v != 0) v = v * at->colscale;
      cup[(size_t)c + (size_t)ncell * p] = v;
      if (!at->chkind) continue;
      /* hydrogen (:1854-1876); Takeda only for a line without an f value */
      double h = 0;
      if (!cont && at->cfac[p] == 0 && at->chkind[p] == SQ_COLH_TAKEDA) {
        h = nh1[c] * (allen / ne[c]) * at->ion[i] / at->g[i] * ex * sqrt(SQ_AME / SQ_AMH);
        h = h * at->cbbhsc;
      } else if (at->chkind[p] == SQ_COLH_DRAWIN) {
        const double q = SQ_RYDV / dev;
        const double divu = q * q;
        double tmp = 2.0 / u0;
        const double mt = SQ_MU_E * tmp;
        tmp = (1.0 + tmp) / (1.0 + mt * mt);
        h = nh1[c] * at->drawin * divu * tmp * ex * sqt;
        if (cont) {
          h = h * at->cbfhsc;
        } else {
          h = h * f;
          h = h * at->cbbhsc;
        }
      }
      if (h != 0) h = h * at->colscale;
      cup[(size_t)c + (size_t)ncell * (ncol + p)] = h;
    }
    const int r0 = at->chkind ? 2 * ncol : ncol;
    for (int r = 0; r < at->ngrec; r++) {
      const int k = at->gcoll ? at->gcoll[r] : -1;
      double u, d;
      sq_gencol_record(at, r, temp[c], ne[c], dxi ? dxi[c] : 0.0, e_kT[c], lsaha ? lsaha[c] : 0.0,
                       nh1 ? nh1[c] : 0.0, k >= 0 ? coll[(size_t)c + (size_t)ncell * k] : 0.0,
                       nstar[(size_t)c + (size_t)ncell * at->gll[r]], nstar[(size_t)c + (size_t)ncell * at->gul[r]],
                       &u, &d);
      cup[(size_t)c + (size_t)ncell * (r0 + r)] = u;
      cup[(size_t)c + (size_t)ncell * (r0 + at->ngrec + r)] = d;
    }
  }
}

/* ---- dense solves of a column-major n x n matrix, a(i,j) = a[i + n*j] ---- */
#define A(i, j) a[(i) + n * (j)]

/* lineq_no_pivot (op_math_mod.f90:420-449).  eqsyst (:365-413) performs the same
 * roundings in the same order with the multipliers negated, so it shares this. */
void sq_lineq_no_pivot(double *a, double *b, int n)
{
  for (int k = 0; k < n - 1; k++) {
    for (int i = k + 1; i < n; i++) A(i, k) = A(i, k) / A(k, k);
    for (int j = k + 1; j < n; j++)
      if (A(k, j) != 0)
        for (int i = k + 1; i < n; i++) A(i, j) = A(i, j) - A(i, k) * A(k, j);
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < i; j++) b[i] = b[i] - A(i, j) * b[j];
  for (int i = n - 1; i >= 0; i--) {
    for (int j = i + 1; j < n; j++) b[i] = b[i] - A(i, j) * b[j];
    b[i] = b[i] / A(i, i);
  }
}

/* lineq, Gaussian elimination with full pivoting (op_math_mod.f90:263-356) */
void sq_lineq(double *a, double *b, int n)
{
  int icol[64];
  double c[64];
  for (int i = 0; i < n; i++) icol[i] = i;
  int ibeg = 0, jbeg = 0;
  while (ibeg < n - 1) {
    double ama = fabs(A(ibeg, jbeg));
    int ima = ibeg, jma = jbeg;
    for (int i = ibeg; i < n; i++)
      for (int j = jbeg; j < n; j++) {
        if (fabs(A(i, j)) <= ama) continue;
        ama = fabs(A(i, j));
        ima = i;
        jma = j;
      }
    for (int i = 0; i < n; i++) {
      const double t = A(i, jma);
      A(i, jma) = A(i, jbeg);
      A(i, jbeg) = t;
    }
    for (int j = jbeg; j < n; j++) {
      const double t = A(ima, j);
      A(ima, j) = A(ibeg, j);
      A(ibeg, j) = t;
    }
    {
      const double t = b[ima];
      b[ima] = b[ibeg];
      b[ibeg] = t;
    }
    {
      const int it = icol[jbeg];
      icol[jbeg] = icol[jma];
      icol[jma] = it;
    }
    ibeg++;
    jbeg++;
    const int imin = ibeg - 1, jmin = jbeg - 1;
    for (int i = ibeg; i < n; i++) {
      const double quot = A(i, jmin) / A(imin, jmin);
      for (int j = jbeg; j < n; j++) A(i, j) = A(i, j) - quot * A(imin, j);
      b[i] = b[i] - quot * b[imin];
    }
  }
  b[n - 1] = b[n - 1] / A(n - 1, n - 1);
  for (int i = n - 2; i >= 0; i--) {
    for (int j = n - 1; j >= i + 1; j--) b[i] = b[i] - A(i, j) * b[j];
    b[i] = b[i] / A(i, i);
  }
  for (int i = 0; i < n; i++) c[icol[i]] = b[i];
  for (int i = 0; i < n; i++) b[i] = c[i];
}

/* LU with partial (row) pivoting, the solver the rate matrix's conditioning
 * asks for where the no-pivot LU loses digits.  Pivot of column k: the first
 * row of largest |a(i,k)|, i >= k.  The row swap covers the whole row (the
 * stored multipliers too).  Forward substitution runs column by column in
 * ascending j, back substitution column by column in descending j: per row
 * the same order as a row-wise loop with j running away from the diagonal
 * (forward) or towards it (back). */
void sq_lu_partial(double *a, double *b, int n)
{
  for (int k = 0; k < n - 1; k++) {
    int p = k;
    double am = fabs(A(k, k));
    for (int i = k + 1; i < n; i++)
      if (fabs(A(i, k)) > am) {
        am = fabs(A(i, k));
        p = i;
      }
    if (p != k) {
      for (int j = 0; j < n; j++) {
        const double t = A(k, j);
        A(k, j) = A(p, j);
        A(p, j) = t;
      }
      const double t = b[k];
      b[k] = b[p];
      b[p] = t;
    }
    for (int i = k + 1; i < n; i++) A(i, k) = A(i, k) / A(k, k);
    for (int j = k + 1; j < n; j++)
      for (int i = k + 1; i < n; i++) A(i, j) = A(i, j) - A(i, k) * A(k, j);
  }
  for (int j = 0; j < n; j++)
    for (int i = j + 1; i < n; i++) b[i] = b[i] - A(i, j) * b[j];
  for (int j = n - 1; j >= 0; j--) {
    b[j] = b[j] / A(j, j);
    for (int i = 0; i < j; i++) b[i] = b[i] - A(i, j) * b[j];
  }
}
#undef A

/* setup_transition_matrix of one cell (atom_mod.f90:740-841) with
 * line_rate_coefficients (:862-884).  bl, ns: b and n* of the cell; gij, gji:
 * the cell's gamma_ij / gamma_ji per transition; cupc: the cell's upward
 * collision rate per pair, electrons then (with chkind) hydrogen, as
 * or_collisions lays them out (unused when cswitch == 0).  Returns W in w
 * (column-major) and the right-hand side in e. */
void or_rate_matrix(const sq_atom_t *at, const sq_params_t *pr, const double *bl, const double *ns, double totn,
                    double ekt, const float *gij, const float *gji, const double *cupc, double *w, double *e)
{
  const int n = at->nlevel;
#define W(i, j) w[(i) + n * (j)]
  memset(w, 0, sizeof(double) * n * n);
  for (int k = 0; k < n; k++) e[k] = 0;
  for (int kr = 0; kr < at->nrad; kr++) {
    if (at->active && !at->active[kr]) continue;
    const int i = at->ti[kr], j = at->tj[kr];
    if ((at->ev[j] - at->ev[i]) * ekt > at->cut_x) {
      const double cut_rate = kr < at->nline ? at->Aji[kr] : at->bf_cut_rate;
      W(i, j) = W(i, j) + cut_rate;
      W(j, i) = W(j, i) + cut_rate * ns[j] / ns[i];
      continue;
    }
    double r_up, r_down;
    const double th = gij[kr], dv = gji[kr];
    if (kr < at->nline) {
      const double g_ij = at->g[i] / at->g[j];
      if (ns[i] > 0 && ns[j] > 0) {
        const double beta_ref = ns[j] * g_ij / ns[i];
        r_up = th * (beta_ref / (1.0 - beta_ref)) + dv;
        r_down = g_ij * (th / (1.0 - beta_ref) + dv);
      } else {
        r_up = 0;
        r_down = 0;
      }
    } else {
      r_up = th;
      r_down = dv;
    }
    W(j, i) = W(j, i) + r_up;
    W(i, j) = W(i, j) + r_down;
  }
  if (pr->cswitch > 0) {
    /* collision_rates (:918-930): c = 0; classic_col adds each nonzero rate,
     * c(j,i) += cup and c(i,j) += cup * n*_i/n*_j, electrons first, then hydrogen
     * (:1846-1876); gencol adds every record's rates (:2350-2351); then w += c *
     * cswitch over the whole matrix (:806-811) */
    double *cm = (double *)calloc((size_t)n * n, sizeof(double));
#define CM(i, j) cm[(i) + n * (j)]
    for (int p = 0; p < at->ncol; p++) {
      const int i = at->ci[p], j = at->cj[p];
      const double nij = ns[i] / ns[j];
      const double ue = cupc[p];
      if (ue != 0) {
        CM(j, i) = CM(j, i) + ue;
        CM(i, j) = CM(i, j) + ue * nij;
      }
      if (at->chkind) {
        const double uh = cupc[at->ncol + p];
        if (uh != 0) {
          CM(j, i) = CM(j, i) + uh;
          CM(i, j) = CM(i, j) + uh * nij;
        }
      }
    }
    const int r0 = at->chkind ? 2 * at->ncol : at->ncol;
    for (int r = 0; r < at->ngrec; r++) {
      const int ll = at->gll[r], ul = at->gul[r];
      CM(ul, ll) = CM(ul, ll) + cupc[r0 + r];
      CM(ll, ul) = CM(ll, ul) + cupc[r0 + at->ngrec + r];
    }
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) W(i, j) = W(i, j) + CM(i, j) * pr->cswitch;
#undef CM
    free(cm);
  }
  for (int i = 0; i < n; i++) {
    double s = 0;
    for (int k = 0; k < n; k++) s = s + W(k, i);
    W(i, i) = -s;
  }
  int pos = 0;
  double best = bl[0] * ns[0];
  for (int k = 1; k < n; k++)
    if (bl[k] * ns[k] > best) {
      best = bl[k] * ns[k];
      pos = k;
    }
  e[pos] = totn;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) W(i, j) = (W(i, j) * bl[j]) * ns[j];
  for (int j = 0; j < n; j++) W(pos, j) = bl[j] * ns[j];
#undef W
}

/* update_populations (atom_mod.f90:439-732) over ncell cells.  A cell whose
 * solution is not finite is left unchanged and reported (the reference stops
 * the run there). */
int or_stateq_update(const sq_atom_t *at, const sq_params_t *pr, int ncell, double *b, const double *nstar,
                     const double *totn, const double *temp, const double *e_kT, const float *gamma_ij,
                     const float *gamma_ji, const double *cup, sq_result_t *res, double *lvlerr)
{
  const int n = at->nlevel, nrad = at->nrad;
  double *w = (double *)malloc(sizeof(double) * n * n);
  const int ncup = (at->chkind ? 2 * at->ncol : at->ncol) + 2 * at->ngrec;
  double *cupc = (double *)malloc(sizeof(double) * (ncup > 0 ? ncup : 1));
  float *gij = (float *)malloc(sizeof(float) * (nrad > 0 ? nrad : 1));
  float *gji = (float *)malloc(sizeof(float) * (nrad > 0 ? nrad : 1));
  double e[64], bl[64], ns[64], bold[64];
  const double eup = fmax(pr->max_update, 1.0), elo = 1.0 / eup;
  res->maxerr = 0;
  res->epos_cell = -1;
  res->epos_level = -1;
  res->nclamp = 0;
  res->ntot = 0;
  res->nonfinite_cell = -1;
  for (int k = 0; k < n; k++) lvlerr[k] = 0;
  for (int c = 0; c < ncell; c++) {
    if (!(totn[c] > 0)) continue;
    if (temp && !(temp[c] < pr->tmax_update)) continue;
    for (int k = 0; k < n; k++) {
      bl[k] = b[(size_t)c + (size_t)ncell * k];
      ns[k] = nstar[(size_t)c + (size_t)ncell * k];
    }
    for (int kr = 0; kr < nrad; kr++) {
      gij[kr] = gamma_ij[(size_t)c + (size_t)ncell * kr];
      gji[kr] = gamma_ji[(size_t)c + (size_t)ncell * kr];
    }
    if (pr->cswitch > 0)
      for (int p = 0; p < ncup; p++) cupc[p] = cup[(size_t)c + (size_t)ncell * p];
    or_rate_matrix(at, pr, bl, ns, totn[c], e_kT[c], gij, gji, cupc, w, e);
    if (pr->solver == 0) sq_lineq_no_pivot(w, e, n);
    else if (pr->solver == 1) sq_lineq(w, e, n);
    else sq_lu_partial(w, e, n);
    int finite = 1;
    for (int k = 0; k < n; k++)
      if (!(fabs(e[k]) <= DBL_MAX)) finite = 0;
    if (!finite) {
      if (res->nonfinite_cell < 0) res->nonfinite_cell = c;
      continue;
    }
    /* the limiter (:596-603), then under-relaxation (:610-612) */
    for (int k = 0; k < n; k++) {
      if (e[k] < elo || e[k] > eup) res->nclamp++;
      res->ntot++;
      if (e[k] < elo) e[k] = elo * exp(fmax(e[k], 0.0) / elo - 1.0);
      else if (e[k] > eup) e[k] = eup * (2.0 - eup / e[k]);
    }
    if (pr->sor_w != 1.0)
      for (int k = 0; k < n; k++) e[k] = pow(e[k], pr->sor_w);
    for (int k = 0; k < n; k++) {
      bold[k] = bl[k];
      bl[k] = bl[k] * e[k];
    }
    double sum = 0;
    for (int k = 0; k < n; k++) sum = sum + bl[k] * ns[k];
    const double norm = totn[c] / sum;
    for (int k = 0; k < n; k++) bl[k] = bl[k] * norm;
    for (int k = 0; k < n; k++)
      if (ns[k] > 0) bl[k] = fmax(bl[k], fmin(1.0, pr->min_pop_frac * totn[c] / ns[k]));
    int imax = 0;
    double wmax = -1;
    for (int k = 0; k < n; k++) {
      e[k] = bold[k] > 0 ? bl[k] / bold[k] - 1.0 : 0.0;
      if (fabs(e[k]) > fabs(lvlerr[k])) lvlerr[k] = e[k];
      double ew = fabs(e[k]);
      if (pr->conv_pop_floor > 0) ew = ew * fmin(1.0, bl[k] * ns[k] / (pr->conv_pop_floor * totn[c]));
      if (ew > wmax) {
        wmax = ew;
        imax = k;
      }
    }
    if (wmax > fabs(res->maxerr)) {
      res->maxerr = copysign(wmax, e[imax]);
      res->epos_cell = c;
      res->epos_level = imax;
    }
    for (int k = 0; k < n; k++) b[(size_t)c + (size_t)ncell * k] = bl[k];
  }
  free(w);
  free(cupc);
  free(gij);
  free(gji);
  return res->nonfinite_cell >= 0 ? 5 : 0;
}

/* ng_accumulate (ng_mod.f90:241-287): gram = d01, d02, d11, d12, d21, d22 and
 * |d0|^2, sums in (cell, level) order with the level fastest; oldb holds the
 * iterates n1, n2, n3 as three consecutive (cell, level) blocks */
void or_ng_accumulate(int ncell, int nlevel, const double *b, const double *oldb, double *gram)
{
  const size_t nv = (size_t)ncell * nlevel;
  double d01 = 0, d02 = 0, d11 = 0, d12 = 0, d22 = 0, s = 0;
  for (int c = 0; c < ncell; c++)
    for (int k = 0; k < nlevel; k++) {
      const size_t idx = (size_t)c + (size_t)ncell * k;
      const double n1 = log(oldb[idx]), n2 = log(oldb[idx + nv]), n3 = log(oldb[idx + 2 * nv]), n4 = log(b[idx]);
      const double d0 = n4 - n3, d1 = d0 - (n3 - n2), d2 = d0 - (n2 - n1);
      d01 = d01 + d0 * d1;
      d02 = d02 + d0 * d2;
      d11 = d11 + d1 * d1;
      d12 = d12 + d1 * d2;
      d22 = d22 + d2 * d2;
      s = s + d0 * d0;
    }
  gram[0] = d01;
  gram[1] = d02;
  gram[2] = d11;
  gram[3] = d12;
  gram[4] = d12;
  gram[5] = d22;
  gram[6] = s;
}

/* ng_extrapolate (ng_mod.f90:314-390): returns 1 when applied, 0 when vetoed */
int or_ng_extrapolate(int ncell, int nlevel, double *b, const double *oldb, const double *nstar, const double *totn,
                      double a, double bc, double max_change, double *emax, long long *epos_cell, int *epos_level)
{
  const size_t nv = (size_t)ncell * nlevel;
  double worst = 0;
  for (int c = 0; c < ncell; c++)
    for (int k = 0; k < nlevel; k++) {
      const size_t idx = (size_t)c + (size_t)ncell * k;
      const double n2 = log(oldb[idx + nv]), n3 = log(oldb[idx + 2 * nv]), n4 = log(b[idx]);
      const double e = (1.0 - a - bc) * n4 + a * n3 + bc * n2;
      worst = fmax(worst, fabs(e - n4));
    }
  *emax = 0;
  *epos_cell = -1;
  *epos_level = -1;
  if (!(exp(worst) - 1.0 <= max_change && fabs(a) <= DBL_MAX && fabs(bc) <= DBL_MAX)) return 0;
  for (int c = 0; c < ncell; c++) {
    for (int k = 0; k < nlevel; k++) {
      const size_t idx = (size_t)c + (size_t)ncell * k;
      const double n2 = log(oldb[idx + nv]), n3 = log(oldb[idx + 2 * nv]), n4 = log(b[idx]);
      const double e = (1.0 - a - bc) * n4 + a * n3 + bc * n2;
      b[idx] = exp(e);
      const double enew = exp(e - n4) - 1.0;
      if (fabs(enew) > fabs(*emax)) {
        *emax = enew;
        *epos_cell = c;
        *epos_level = k;
      }
    }
    double s = 0;
    for (int k = 0; k < nlevel; k++) s = s + b[(size_t)c + (size_t)ncell * k] * nstar[(size_t)c + (size_t)ncell * k];
    const double f = totn[c] / s;
    for (int k = 0; k < nlevel; k++) b[(size_t)c + (size_t)ncell * k] = b[(size_t)c + (size_t)ncell * k] * f;
  }
  return 1;
}

/*
 * or_hprof.c -- CPU restatement of the analytic hydrogen line profiles of
 * HOP/hprofl_mod.f90 (after HLINOP): hydrogen_line, hfnm, hcell_prepare,
 * stark_prepare/stark_eval with holtsmark and vcse1f, hvoigt, lyman_voigt,
 * classical_wing, lyman_interp, and the outward frequency walk of
 * add_h_opacities.  TEST INFRASTRUCTURE ONLY.
 *
 * Kinds follow the Fortran declarations: a default-real literal or variable is
 * float, a real(8) one double, and a mixed expression is evaluated in double and
 * rounded where the Fortran assigns it to a real(4).  Integer powers are the
 * multiplication chains the compiler forms (x**2 = x*x, x**3 = (x*x)*x,
 * x**4 = (x*x)*(x*x)).  Nothing is contracted (-ffp-contract=off).
 */
#include "or_hprof.h"

#include <float.h>
#include <math.h>
#include <stddef.h>

#include "or_htables.inc"
#include "or_vcs.h"

void or_qlg_coef(float a, float c[5]);
float or_qlg_eval(const float *tgx, const float *th2x, const float c[5], float v);

static const double H_PI = 3.14159265359, H_EULER = 0.5772156649;
static const double H_CC = 2.99792458e10, H_HH = 6.626176e-27, H_BK = 1.380662e-16;
#define H_HK (H_HH / H_BK)
#define H_OVER_4PI (1.0 / (4.0 * H_PI))
static const double H_LAM_LYRAY = 1400.0;
#define H_LYA0 ((double)82259.105f)
#define H_REDTHRESH (20000.0 / H_LYA0 - 1.0)
#define H_Q4000 (-4000.0 / H_LYA0)

/* hfnm (hprofl_mod.f90:845-888): absorption oscillator strength n -> m */
static double hfnm(int n, int m)
{
  if (m <= n) return 0.0;
  const double xn = n, xm = m;
  const double ginf = (double)(0.2027f / powf((float)n, 0.71f));
  const double gca = (double)(0.124f / (float)n);
  const double fkn = (double)((float)n * 1.9603f);
  const double wtc = (double)(0.45f - 2.4f / (float)(n * n * n) * ((float)n - 1.0f));
  const double xmn = (double)(m - n);
  const double t = xm / (xmn * (double)(m + n));
  const double fk = fkn * ((t * t) * t);
  const double xmn12 = pow(xmn, (double)1.2f);
  const double wt = (xmn12 - 1.0) / (xmn12 + wtc);
  (void)xn;
  return fk * (1.0 - wt * ginf - ((double)0.222f + gca / xm) * (1.0 - wt));
}

/* hydrogen_line (hprofl_mod.f90:703-810) */
void or_hydrogen_line(int n, int m, double nu0, unsigned opts, or_hline_t *h)
{
  const int mmn = m - n, n2 = n * n, m2 = m * m;
  const float mn2 = (float)(m2 * n2);
  const float ignm = mn2 / (float)(m2 - n2);
  for (int i = 0; i < 14; i++) h->dq[i] = h->wt[i] = 0.0;
  h->n = n;
  h->m = m;
  h->nu0 = nu0;
  h->bpo = 0;
  h->opts = (int)opts;
  h->pad = 0;
  h->qray = -HUGE_VAL;
  float xknm;
  if (mmn <= 3 && n <= 4) xknm = H_XKNM[(mmn - 1) * 4 + (n - 1)];
  else xknm = ((5.5e-5f * ignm) * mn2) / (1.0f + 0.13f / (float)mmn);
  h->gstk = ((double)(5.0f * xknm) * nu0) / (H_CC * (double)1e8f);
  const float radamp = n == 1 ? H_ASUMLY[m - 1] : H_ASUM[n - 1] + H_ASUM[m - 1];
  h->grad = ((double)radamp * H_OVER_4PI) / nu0;
  if (n == 1) h->qray = (H_CC * 1e8) / (H_LAM_LYRAY * nu0) - 1.0;
  float resont;
  if (n != 1) resont = (float)(hfnm(1, n) / (double)(1.0f - 1.0f / (float)n2));
  else resont = (float)(hfnm(1, m) / (double)(1.0f - 1.0f / (float)m2));
  h->gw1 = (double)((resont * 2.07e-24f) * ignm);
  h->gw2 = 0.0;
  if (!(opts & 8) && n == 2 && m <= 5) {
    static const float sigma[3] = {3.304e-18f * 1.e4f, 6.497e-18f * 1.e4f, 1.178e-17f * 1.e4f};
    static const float alf[3] = {0.677f, 0.455f, 0.380f};
    static const float balfac[3] = {0.97875f * 1.e6f, 0.97659f * 1.e6f, 0.97794f * 1.e6f};
    resont = balfac[mmn - 1] * sigma[mmn - 1];
    h->gw2 = (double)(0.5f * (1.0f - alf[mmn - 1]));
    h->gw1 = ((double)resont * pow((double)1e-12f, h->gw2)) / ((nu0 * 2.0) * H_PI);
    h->bpo = 1;
  }
  h->gw3 = (double)((4.45e-26f * ignm) * powf((float)m2 * (7.0f * (float)m2 + 5.0f), 0.4f));
  static const int istal[4] = {1, 3, 10, 21}, lnghal[4] = {2, 7, 11, 14}, lncomp[4] = {1, 3, 4, 5};
  int ifins;
  double finest[14], finswt[14];
  if (n > 4 || m > 10) {
    ifins = 1;
    finest[0] = 0.0;
    finswt[0] = 1.0;
  } else if (m - n > 1) {
    ifins = lncomp[n - 1];
    for (int i = 0; i < ifins; i++) {
      finest[i] = (double)(H_STCOMP[(n - 1) * 5 + i] * 1e7f);
      finswt[i] = (double)(H_STCPWT[(n - 1) * 5 + i] / (float)(n * n));
    }
  } else {
    ifins = lnghal[n - 1];
    const int ipos = istal[n - 1];
    for (int i = 0; i < ifins; i++) {
      const int k = ipos - 1 + i;
      finest[i] = (double)(H_STALPH[k] * 1e7f);
      finswt[i] = (double)(H_STWTAL[k] / (float)(3 * n * n));
    }
  }
  h->io = ifins;
  double dqbar = 0.0, dqmax = 0.0;
  for (int i = 0; i < ifins; i++) {
    h->dq[i] = finest[i] / nu0;
    h->wt[i] = finswt[i];
    dqbar = dqbar + h->wt[i] * h->dq[i];
    dqmax = fmax(dqmax, fabs(h->dq[i]));
  }
  h->dqbar = dqbar;
  h->dqmax = dqmax;
  if (opts & 1) h->grad = 0.0;
  if (opts & 2) h->gstk = 0.0;
  if (opts & 4) {
    h->gw1 = h->gw2 = h->gw3 = 0.0;
    h->bpo = 0;
  }
}

/* vcse1f (hprofl_mod.f90:1205-1219) */
static double vcse1f(double x)
{
  if (x <= 0.0) return 0.0;
  if (x <= (double)0.01f) return -log(x) - H_EULER + x;
  if (x <= 1.0)
    return -log(x) - H_EULER +
           x * ((double)0.99999193f +
                x * ((double)-0.24991055f +
                     x * ((double)0.05519968f + x * ((double)-0.00976004f + x * (double)0.00107857f))));
  if (x <= 30.0)
    return (x * (x + (double)2.334733f) + (double)0.25062f) / (x * (x + (double)3.330657f) + (double)1.681534f) / x *
           exp(-x);
  return 0.0;
}

/* holtsmark (hprofl_mod.f90:1029-1199): a default-real result */
static float holtsmark(double b, double p, int n, int m)
{
  const double b2 = b * b, sb = sqrt(b);
  if (b > 500.0) return (float)(((double)1.5f / sb + 27.0 / b2) / b2);
  double corr;
  int indx = 7;
  const int mmn = m - n;
  if (n <= 3 && mmn <= 2) indx = 2 * (n - 1) + mmn;
  const float *prob = H_PROB[indx - 1];
  int im = (int)(5.0 * p) + 1;
  if (im > 4) im = 4;
  const int ip = im + 1;
  const double wtpp = 5.0 * (p - (double)H_PP[im - 1]);
  const double wtpm = 1.0 - wtpp;
  if (b <= (double)25.12f) {
    int jp = 2;
    while (b > (double)H_BETA[jp - 1] && jp < 15) jp++;
    const int jm = jp - 1;
    const double wtbp = (b - (double)H_BETA[jm - 1]) / (double)(H_BETA[jp - 1] - H_BETA[jm - 1]);
    const double wtbm = 1.0 - wtbp;
#define PB(i, j) ((double)prob[((i)-1) + 5 * ((j)-1)])
    const double cbp = PB(ip, jp) * wtpp + PB(im, jp) * wtpm;
    const double cbm = PB(ip, jm) * wtpp + PB(im, jm) * wtpm;
#undef PB
    corr = 1.0 + cbp * wtbp + cbm * wtbm;
    double pr1 = 0.0, pr2 = 0.0;
    const double wt = fmax(fmin((double)0.5f * (10.0 - b), 1.0), 0.0);
    if (b <= 10.0) pr1 = 8.0 / (83.0 + (2.0 + (double)0.95f * b2) * b);
    if (b >= 8.0) pr2 = ((double)1.5f / sb + 27.0 / b2) / b2;
    return (float)((pr1 * wt + pr2 * (1.0 - wt)) * corr);
  }
  const double cc = (double)H_HC[indx - 1][ip - 1] * wtpp + (double)H_HC[indx - 1][im - 1] * wtpm;
  const double dd = (double)H_HD[indx - 1][ip - 1] * wtpp + (double)H_HD[indx - 1][im - 1] * wtpm;
  corr = 1.0 + dd / (cc + b * sb);
  return (float)(((double)1.5f / sb + 27.0 / b2) / b2 * corr);
}

typedef struct {
  int off, n, m;
  double hw5, pp, cne, ex, c1coef, g1, gcon1, gcon2, gam0;
} stark_t;

/* stark_prepare (hprofl_mod.f90:892-966) */
static void stark_prepare(int n, int m, double nu0, float temp, float ne, float hwstk, stark_t *s)
{
  s->off = hwstk == 0.0f;
  if (s->off) return;
  s->n = n;
  s->m = m;
  s->hw5 = (double)hwstk * 0.2;
  const double t4 = (double)temp * 1e-4;
  const double xne16 = pow((double)ne, 0.1666667);
  s->pp = xne16 * 0.08989 / sqrt((double)temp);
  s->cne = sqrt(5.96e-23 * (double)ne);
  const double y1b = 2.0 / (1.0 + 0.012 / (double)temp * (double)sqrtf(ne / temp));
  const double y1s = pow(t4, 0.3) / xne16;
  s->gcon1 = 0.2 + 0.09 * sqrt(t4) / (1.0 + (double)ne * 1e-13);
  s->gcon2 = 0.2 / (1.0 + (double)ne * 1e-15);
  const double gcon = 1.0 - s->gcon1 - s->gcon2;
  const int mmn = m - n;
  const double xm2mn2 = (double)(m * m - n * n);
  const double y1num = m == 2 ? 550.0 : (m == 3 ? 380.0 : 320.0);
  static const float y1wtm[2][2] = {{1.e18f, 1.e17f}, {1.e16f, 1.e14f}};   /* [mmn-1][n-1] */
  double y1wht;
  if (mmn <= 2 && n <= 2) y1wht = (double)y1wtm[mmn - 1][n - 1];
  else if (mmn <= 3) y1wht = 1e14;
  else y1wht = 1e13;
  const double wty1 = 1.0 / (1.0 + (double)ne / y1wht);
  const double y1scal = y1num * y1s * wty1 + y1b * (1.0 - wty1);
  s->ex = H_HK * nu0 / (double)temp;
  s->c1coef = 0.5 * y1scal * s->ex * xm2mn2;
  const double c1 = s->hw5 * s->c1coef;
  s->g1 = 6.77 * sqrt(c1);
  s->gam0 = s->g1 * fmax(0.0, 0.2114 - log(c1 * s->cne)) * gcon;
}

/* stark_eval (hprofl_mod.f90:969-1021) */
static double stark_eval(const stark_t *s, double q)
{
  if (s->off) return 0.0;
  const double q1 = fabs(q);
  const double y1 = s->c1coef * q1;
  const double t = q1 / s->cne;
  const double y2 = t * t;
  const double beta = q1 / s->hw5;
  double gam;
  if (y2 <= 1e-4 && y1 <= 1e-5) {
    gam = s->gam0;
  } else {
    const double u = 90.0 * y1;
    gam = s->g1 * (0.5 * exp(-fmin(80.0, y1)) + vcse1f(y1) - 0.5 * vcse1f(y2)) *
          (1.0 - s->gcon1 / (1.0 + (u * u) * u) - s->gcon2 / (1.0 + 2000.0 * y1));
    if (gam <= 1e-20) gam = 0.0;
  }
  const double prqs = (double)holtsmark(beta, s->pp, s->n, s->m);
  const double f = gam > 0.0 ? gam / H_PI / (gam * gam + beta * beta) : 0.0;
  const double v = 0.9 * y1;
  const double p1 = v * v;
  const double fns = (p1 + 0.03 * sqrt(y1)) / (p1 + 1.0);
  double stark = (prqs * (1.0 + fns) + f) / s->hw5;
  if (q < 0.0) stark = stark * exp(s->ex * q);
  return stark;
}

/* classical_wing (hprofl_mod.f90:544-549) */
static float classical_wing(double q)
{
  const double a = 1.0 + q, b = 2.0 + q;
  const double a2 = a * a;
  return (float)(4.0 * (a2 * a2) / (b * b));
}

/* lyman_interp (hprofl_mod.f90:829-842) on a table of n values */
static double lyman_interp(const float *tab, int n, float dx, float x0, double newx)
{
#define LV(k) ((double)(tab[(k)] - 14.0f))
  const double x = (newx - (double)x0) / (double)dx;
  int i = (int)fmax(0.0, x);
  if (i > n - 2) i = n - 2;
  return (LV(i + 1) - LV(i)) * (x - (double)i) + LV(i);
#undef LV
}

typedef struct {
  float idf, ne, tothi, resont, vdw, hwstk, hwlor, hfwid;
  float hwadd;
  int use_vcs;
  or_vcs_cell_t vcs;
  int lymanalf;
  stark_t st;
  float vcore[5], vwing[5], vwing_ray[5];
  double xholt4000;
} hcell_t;

/* hcell_prepare (hprofl_mod.f90:388-438), the analytic branch */
static void hcell_prepare(const or_hline_t *h, float temp, float ne, float fo, float vbar2h, float tothi, float t3nhe,
                          float idf, hcell_t *c)
{
  c->idf = idf;
  c->ne = ne;
  c->tothi = tothi;
  c->resont = (float)((double)tothi * h->gw1);
  if (h->gw2 != 0.0) c->resont = (float)((double)c->resont * pow((double)vbar2h, h->gw2));
  c->hwstk = (float)(h->gstk * (double)fo);
  c->vdw = (float)(h->gw3 * (double)t3nhe);
  c->hwlor = (float)(h->grad + (double)c->resont + (double)c->vdw);
  c->hfwid = fmaxf(fmaxf(1.0f / idf, c->hwlor), c->hwstk);
  c->hwadd = 0.0f;
  c->use_vcs = or_vcs_supported(h->n, h->m);
  if (c->use_vcs) {
    /* the tabulated profile, with the broadening the table lacks added as one
     * Lorentzian (hprofl_mod.f90:412-426) */
    c->hwadd = c->vdw;
    if (!or_vcs_radiative(h->n)) c->hwadd = c->hwadd + (float)h->grad;
    if (h->bpo || !or_vcs_resonance(h->n, h->m)) c->hwadd = c->hwadd + c->resont;
    float nh_table = tothi;
    if (h->bpo || (h->opts & 4)) nh_table = 0.0f;
    c->hfwid = fmaxf(1.0f / idf, c->hwadd);
    or_vcs_prepare(h->n, h->m, h->nu0, temp, ne, nh_table, &c->vcs);
    c->lymanalf = 0;
    return;
  }
  c->lymanalf = h->n == 1 && h->m == 2;
  stark_prepare(h->n, h->m, h->nu0, temp, ne, c->hwstk, &c->st);
  or_qlg_coef((c->hwlor + c->hwstk) * idf, c->vcore);
  or_qlg_coef(c->hwlor * idf, c->vwing);
  if (h->n == 1) or_qlg_coef((c->resont + c->vdw) * idf, c->vwing_ray);
  c->xholt4000 = c->lymanalf ? 0.5 * stark_eval(&c->st, H_Q4000) : 0.0;
}

/* hvoigt (hprofl_mod.f90:465-499) */
static float hvoigt(const float *tgx, const float *th2x, const or_hline_t *h, const hcell_t *c, double q)
{
  float phi;
  if (fabs(q) > (double)c->hfwid) {
    phi = (float)stark_eval(&c->st, q);
    const float *vw = q < h->qray ? c->vwing_ray : c->vwing;
    float wing = 0.0f;
    for (int i = 0; i < h->io; i++) {
      const float vs = (float)((q - h->dq[i]) * (double)c->idf);
      const float xv = or_qlg_eval(tgx, th2x, vw, vs) * c->idf;
      wing = (float)((double)wing + h->wt[i] * (double)xv);
    }
    phi = phi + classical_wing(q) * wing;
  } else {
    phi = 0.0f;
    for (int i = 0; i < h->io; i++) {
      const float vs = (float)((q - h->dq[i]) * (double)c->idf);
      const float xv = or_qlg_eval(tgx, th2x, c->vcore, vs) * c->idf;
      phi = (float)((double)phi + h->wt[i] * (double)xv);
    }
  }
  return phi;
}

/* lyman_voigt (hprofl_mod.f90:582-692) */
static float lyman_voigt(const float *tgx, const float *th2x, const or_hline_t *h, const hcell_t *c, double q)
{
  float vcw[5];
  const float *vc = c->vcore;
  const int wing = fabs(q) > (double)c->hfwid;
  if (wing) {
    float a = 0.0f;
    if (q > h->qray) a = (float)(h->grad * (double)classical_wing(q));
    if (q > H_Q4000) {
      float xfac = 1.0f;
      if (q < 0.0) xfac = (float)((double)xfac + (double)0.13f * q / H_Q4000);
      a = a + xfac * c->resont + c->vdw;
    }
    or_qlg_coef(a * c->idf, vcw);
    vc = vcw;
  }
  float phi = 0.0f;
  for (int i = 0; i < h->io; i++) {
    const float vs = (float)((q - h->dq[i]) * (double)c->idf);
    const float xv = or_qlg_eval(tgx, th2x, vc, vs) * c->idf;
    phi = (float)((double)phi + h->wt[i] * (double)xv);
  }
  if (wing && q > H_REDTHRESH) {
    if (q <= H_Q4000) {
      float x = (float)lyman_interp(H_LYH2, 91, 200.0f, -22000.0f, q * H_LYA0);
      phi = (float)((double)phi + H_LYA0 * (double)c->tothi * (double)powf(10.0f, x));
      x = (float)lyman_interp(H_LYH2PLUS, 111, 100.0f, -15000.0f, q * H_LYA0);
      phi = (float)((double)phi + H_LYA0 * (double)c->ne * (double)powf(10.0f, x));
      phi = (float)((double)phi + (double)0.5f * stark_eval(&c->st, q));
    } else {
      double xstark = (double)0.5f * stark_eval(&c->st, q);
      if (q < 0.0 && xstark > 0.0 && c->xholt4000 > 0.0) {
        const double sat4000 = H_LYA0 * (double)c->ne * pow(10.0, (double)(H_LYH2PLUS[110] - 14.0f));
        const float xfac = (float)(1.0 + (sat4000 / c->xholt4000 - 1.0) * q / H_Q4000);
        xstark = xstark * (1.0 + (double)xfac);
      }
      phi = (float)((double)phi + xstark);
    }
  }
  return phi;
}

/* added_wing (hprofl_mod.f90:560-574) */
static float added_wing(const hcell_t *c, double d)
{
  if (fabs(d) > (double)c->hfwid)
    return (float)((double)c->hwadd / (H_PI * (d * d + (double)c->hwadd * (double)c->hwadd))) * classical_wing(d);
  return 0.0f;
}

/* vcs_fine (hprofl_mod.f90:514-536) */
static float vcs_fine(const or_hline_t *h, const hcell_t *c, double q)
{
  float phi;
  if (fabs(q) - h->dqmax > c->vcs.q_tail) {
    phi = (float)or_vcs_tail(&c->vcs, log(fabs(q - h->dqbar)));
    if (c->hwadd > 0.0f) phi = phi + added_wing(c, q - h->dqbar);
    return phi;
  }
  phi = 0.0f;
  for (int i = 0; i < h->io; i++) phi = (float)((double)phi + h->wt[i] * (double)(float)or_vcs_eval(&c->vcs, q - h->dq[i]));
  if (c->hwadd > 0.0f)
    for (int i = 0; i < h->io; i++) phi = (float)((double)phi + h->wt[i] * (double)added_wing(c, q - h->dq[i]));
  return phi;
}

static float hprofile(const float *tgx, const float *th2x, const or_hline_t *h, const hcell_t *c, double q)
{
  if (c->use_vcs) return vcs_fine(h, c, q);
  return c->lymanalf ? lyman_voigt(tgx, th2x, h, c, q) : hvoigt(tgx, th2x, h, c, q);
}

/* profile_at (hprofl_mod.f90:336-350): past qt every component is on the table's
 * power-law tail, evaluated from ln|d| of the rest-frame detuning and the shift */
static float profile_at(const float *tgx, const float *th2x, const or_hline_t *h, const hcell_t *c, double qt,
                        double vp, double nu_f, double q)
{
  if (fabs(q) > qt) {
    double d = (nu_f - h->nu0) / h->nu0 - h->dqbar;
    d = copysign(fmax(fabs(d), DBL_MIN), d);
    const double lnd = log(fabs(d)), invd = 1.0 / d;
    const double r = vp * invd;
    float phi = (float)or_vcs_tail(&c->vcs, lnd - r * (1.0 + 0.5 * r));
    if (c->hwadd > 0.0f) phi = phi + added_wing(c, q - h->dqbar);
    return phi;
  }
  return hprofile(tgx, th2x, h, c, q);
}

void or_hprofile(const or_hline_t *h, const float *tgx, const float *th2x, float temp, float ne, float fo,
                 float vbar2h, float tothi, float t3nhe, float idf, int n, const double *q, float *phi)
{
  hcell_t c;
  hcell_prepare(h, temp, ne, fo, vbar2h, tothi, t3nhe, idf, &c);
  for (int i = 0; i < n; i++) phi[i] = hprofile(tgx, th2x, h, &c, q[i]);
}

void or_add_h_opacities(const or_hline_t *h, const float *tgx, const float *th2x, double Bij, int f0, int nf,
                        const double *nu, long long ncell, const or_hcells_t *cl, const float *bi,
                        const float *bj, float *chi, float *eta, const float *cont, int *line_used,
                        float *line_strength)
{
  const float tol = 1e-7f;
  const float inv_nu0 = (float)(1.0 / h->nu0);
  int used = 0;
  float strength = 0.0f;
  for (long long i = 0; i < ncell; i++) {
    const float idf = cl->inv_df[i];
    const float v = (float)((double)(cl->vproj[i] + 1.0f) * h->nu0);
    const float Rij = (float)((double)cl->ni[i] * Bij);
    const float cchi = bi ? Rij * bi[i] : Rij, ceta = bj ? Rij * bj[i] : Rij;
    hcell_t c;
    hcell_prepare(h, cl->temp[i], cl->ne[i], cl->fo[i], cl->vbar2h[i], cl->tothi[i], cl->t3nhe[i], idf, &c);
    const size_t base = (size_t)nf * (size_t)i;
    const double qt = c.use_vcs ? c.vcs.q_tail + h->dqmax : HUGE_VAL;
    const double vp = (double)cl->vproj[i];
    const float ref = tol * cont[base + f0];
    float lchi = ref;
    for (int f = f0; lchi >= ref && f < nf; f++) {
      const double q = (nu[f] - (double)v) * (double)inv_nu0;
      const float phi = profile_at(tgx, th2x, h, &c, qt, vp, nu[f], q);
      lchi = phi * cchi;
      const float leta = phi * ceta;
      chi[base + f] = chi[base + f] + lchi;
      eta[base + f] = eta[base + f] + leta;
      if (f == f0) {
        used = 1;
        strength = fmaxf(strength, lchi / cont[base + f0]);
      }
    }
    lchi = ref;
    for (int f = f0 - 1; lchi >= ref && f >= 0; f--) {
      const double q = (nu[f] - (double)v) * (double)inv_nu0;
      const float phi = profile_at(tgx, th2x, h, &c, qt, vp, nu[f], q);
      lchi = phi * cchi;
      const float leta = phi * ceta;
      chi[base + f] = chi[base + f] + lchi;
      eta[base + f] = eta[base + f] + leta;
    }
  }
  if (used) {
    *line_used = 1;
    *line_strength = fmaxf(*line_strength, strength);
  }
}

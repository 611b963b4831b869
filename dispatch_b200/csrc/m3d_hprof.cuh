// Hydrogen line profiles on the device (HOP/hprofl_mod.f90, after HLINOP), the
// analytic path: the Stark profile of Griem's theory with the VCS-approximating
// corrections (stark_prepare, stark_eval, holtsmark, vcse1f), the fine-structure
// sums of QLG-bot Voigt profiles inside the switch width hfwid and Stark + Lorentz
// outside it (hvoigt), and Lyman alpha's quasi-molecular satellite wings
// (lyman_voigt).  Kinds follow the Fortran declarations: default reals are float,
// real(8) are double, and a mixed expression is evaluated in double and rounded
// where the Fortran assigns it to a real(4).  The line constants (hline_t) come
// from the host's hydrogen_line.
#pragma once
#include "m3d_htables.cuh"
#include "m3d_qlg.cuh"

namespace m3d {

struct HLineDev {
  int n, m, bpo, io;
  double nu0, grad, gstk, gw1, gw2, gw3;
  double dq[14], wt[14];
  double dqbar, dqmax, qray;
};

constexpr double H_PI = 3.14159265359;                    // const_mod.f90:14
constexpr double H_EULER = 0.5772156649;                  // const_mod.f90:15
constexpr double H_LYA0 = (double)82259.105f;             // hprofl_mod.f90:196, a default-real literal
#define H_REDTHRESH (20000.0 / H_LYA0 - 1.0)
#define H_Q4000 (-4000.0 / H_LYA0)

// qlg_bot_coef / qlg_bot_eval (qlg_mod.f90:515-528)
__device__ __forceinline__ QlgCoef h_qlg_coef(float a) { return qlg_setup(a, 1.0f, 0.8325546112f, 1.7724538509f); }
__device__ __forceinline__ float h_qlg_eval(const float2 *tab, const QlgCoef &c, float v) {
  return qlg_eval(tab, c, v) * 0.5641895835f;
}

// vcse1f (hprofl_mod.f90:1205-1219)
__device__ __forceinline__ double h_vcse1f(double x) {
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

// holtsmark (hprofl_mod.f90:1029-1199), a default-real result
__device__ __forceinline__ float h_holtsmark(double b, double p, int n, int m) {
  const double b2 = b * b, sb = sqrt(b);
  if (b > 500.0) return (float)(((double)1.5f / sb + 27.0 / b2) / b2);
  int indx = 7;
  const int mmn = m - n;
  if (n <= 3 && mmn <= 2) indx = 2 * (n - 1) + mmn;
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
    const float *prob = H_PROB[indx - 1];
    const double cbp = (double)prob[(ip - 1) + 5 * (jp - 1)] * wtpp + (double)prob[(im - 1) + 5 * (jp - 1)] * wtpm;
    const double cbm = (double)prob[(ip - 1) + 5 * (jm - 1)] * wtpp + (double)prob[(im - 1) + 5 * (jm - 1)] * wtpm;
    const double corr = 1.0 + cbp * wtbp + cbm * wtbm;
    double pr1 = 0.0, pr2 = 0.0;
    const double wt = fmax(fmin((double)0.5f * (10.0 - b), 1.0), 0.0);
    if (b <= 10.0) pr1 = 8.0 / (83.0 + (2.0 + (double)0.95f * b2) * b);
    if (b >= 8.0) pr2 = ((double)1.5f / sb + 27.0 / b2) / b2;
    return (float)((pr1 * wt + pr2 * (1.0 - wt)) * corr);
  }
  const double cc = (double)H_HC[indx - 1][ip - 1] * wtpp + (double)H_HC[indx - 1][im - 1] * wtpm;
  const double dd = (double)H_HD[indx - 1][ip - 1] * wtpp + (double)H_HD[indx - 1][im - 1] * wtpm;
  const double corr = 1.0 + dd / (cc + b * sb);
  return (float)(((double)1.5f / sb + 27.0 / b2) / b2 * corr);
}

struct HStark {
  int off, n, m;
  double hw5, pp, cne, ex, c1coef, g1, gcon1, gcon2, gam0;
};

// stark_prepare (hprofl_mod.f90:892-966)
__device__ __forceinline__ void h_stark_prepare(int n, int m, double nu0, float temp, float ne, float hwstk,
                                                HStark &s) {
  s.off = hwstk == 0.0f;
  s.n = n;
  s.m = m;
  if (s.off) return;
  s.hw5 = (double)hwstk * 0.2;
  const double t4 = (double)temp * 1e-4;
  const double xne16 = pow((double)ne, 0.1666667);
  s.pp = xne16 * 0.08989 / sqrt((double)temp);
  s.cne = sqrt(5.96e-23 * (double)ne);
  const double y1b = 2.0 / (1.0 + 0.012 / (double)temp * (double)sqrtf(ne / temp));
  const double y1s = pow(t4, 0.3) / xne16;
  s.gcon1 = 0.2 + 0.09 * sqrt(t4) / (1.0 + (double)ne * 1e-13);
  s.gcon2 = 0.2 / (1.0 + (double)ne * 1e-15);
  const double gcon = 1.0 - s.gcon1 - s.gcon2;
  const int mmn = m - n;
  const double xm2mn2 = (double)(m * m - n * n);
  const double y1num = m == 2 ? 550.0 : (m == 3 ? 380.0 : 320.0);
  double y1wht;
  if (mmn <= 2 && n <= 2) {
    // y1wtm(n, mmn) = reshape([1e18, 1e17, 1e16, 1e14], [2,2]), default reals
    const float w = mmn == 1 ? (n == 1 ? 1.e18f : 1.e17f) : (n == 1 ? 1.e16f : 1.e14f);
    y1wht = (double)w;
  } else {
    y1wht = mmn <= 3 ? 1e14 : 1e13;
  }
  const double wty1 = 1.0 / (1.0 + (double)ne / y1wht);
  const double y1scal = y1num * y1s * wty1 + y1b * (1.0 - wty1);
  s.ex = M3D_H_K * nu0 / (double)temp;
  s.c1coef = 0.5 * y1scal * s.ex * xm2mn2;
  const double c1 = s.hw5 * s.c1coef;
  s.g1 = 6.77 * sqrt(c1);
  s.gam0 = s.g1 * fmax(0.0, 0.2114 - log(c1 * s.cne)) * gcon;
}

// stark_eval (hprofl_mod.f90:969-1021)
__device__ __forceinline__ double h_stark_eval(const HStark &s, double q) {
  if (s.off) return 0.0;
  const double q1 = fabs(q);
  const double y1 = s.c1coef * q1;
  const double t = q1 / s.cne;
  const double y2 = t * t;
  const double beta = q1 / s.hw5;
  double gam;
  if (y2 <= 1e-4 && y1 <= 1e-5) {
    gam = s.gam0;
  } else {
    const double u = 90.0 * y1;
    gam = s.g1 * (0.5 * exp(-fmin(80.0, y1)) + h_vcse1f(y1) - 0.5 * h_vcse1f(y2)) *
          (1.0 - s.gcon1 / (1.0 + (u * u) * u) - s.gcon2 / (1.0 + 2000.0 * y1));
    if (gam <= 1e-20) gam = 0.0;
  }
  const double prqs = (double)h_holtsmark(beta, s.pp, s.n, s.m);
  const double f = gam > 0.0 ? gam / H_PI / (gam * gam + beta * beta) : 0.0;
  const double v = 0.9 * y1;
  const double p1 = v * v;
  const double fns = (p1 + 0.03 * sqrt(y1)) / (p1 + 1.0);
  double stark = (prqs * (1.0 + fns) + f) / s.hw5;
  if (q < 0.0) stark = stark * exp(s.ex * q);
  return stark;
}

// classical_wing (hprofl_mod.f90:544-549)
__device__ __forceinline__ float h_classical_wing(double q) {
  const double a = 1.0 + q, b = 2.0 + q;
  const double a2 = a * a;
  return (float)(4.0 * (a2 * a2) / (b * b));
}

// lyman_interp (hprofl_mod.f90:829-842); the tables are default-real literals minus 14
__device__ __forceinline__ double h_lyman_interp(const float *tab, int n, float dx, float x0, double newx) {
  const double x = (newx - (double)x0) / (double)dx;
  int i = (int)fmax(0.0, x);
  if (i > n - 2) i = n - 2;
  const double a = (double)(tab[i] - 14.0f), b = (double)(tab[i + 1] - 14.0f);
  return (b - a) * (x - (double)i) + a;
}

struct HCell {
  float idf, ne, tothi, resont, vdw, hwstk, hwlor, hfwid;
  int lymanalf;
  HStark st;
  QlgCoef vcore, vwing, vwing_ray;
  double xholt4000;
};

// hcell_prepare (hprofl_mod.f90:388-438), the analytic branch
__device__ __forceinline__ void h_cell_prepare(const HLineDev &h, float temp, float ne, float fo, float vbar2h,
                                               float tothi, float t3nhe, float idf, HCell &c) {
  c.idf = idf;
  c.ne = ne;
  c.tothi = tothi;
  c.resont = (float)((double)tothi * h.gw1);
  if (h.gw2 != 0.0) c.resont = (float)((double)c.resont * pow((double)vbar2h, h.gw2));
  c.hwstk = (float)(h.gstk * (double)fo);
  c.vdw = (float)(h.gw3 * (double)t3nhe);
  c.hwlor = (float)(h.grad + (double)c.resont + (double)c.vdw);
  c.hfwid = fmaxf(fmaxf(1.0f / idf, c.hwlor), c.hwstk);
  c.lymanalf = h.n == 1 && h.m == 2;
  h_stark_prepare(h.n, h.m, h.nu0, temp, ne, c.hwstk, c.st);
  c.vcore = h_qlg_coef((c.hwlor + c.hwstk) * idf);
  c.vwing = h_qlg_coef(c.hwlor * idf);
  c.vwing_ray = h.n == 1 ? h_qlg_coef((c.resont + c.vdw) * idf) : c.vwing;
  c.xholt4000 = c.lymanalf ? 0.5 * h_stark_eval(c.st, H_Q4000) : 0.0;
}

// hvoigt (hprofl_mod.f90:465-499)
__device__ __forceinline__ float h_voigt(const float2 *tab, const HLineDev &h, const HCell &c, double q) {
  float phi;
  if (fabs(q) > (double)c.hfwid) {
    phi = (float)h_stark_eval(c.st, q);
    const QlgCoef &vw = q < h.qray ? c.vwing_ray : c.vwing;
    float wing = 0.0f;
    for (int i = 0; i < h.io; i++) {
      const float vs = (float)((q - h.dq[i]) * (double)c.idf);
      const float xv = h_qlg_eval(tab, vw, vs) * c.idf;
      wing = (float)((double)wing + h.wt[i] * (double)xv);
    }
    phi = phi + h_classical_wing(q) * wing;
  } else {
    phi = 0.0f;
    for (int i = 0; i < h.io; i++) {
      const float vs = (float)((q - h.dq[i]) * (double)c.idf);
      const float xv = h_qlg_eval(tab, c.vcore, vs) * c.idf;
      phi = (float)((double)phi + h.wt[i] * (double)xv);
    }
  }
  return phi;
}

// lyman_voigt (hprofl_mod.f90:582-692)
__device__ __forceinline__ float h_lyman_voigt(const float2 *tab, const HLineDev &h, const HCell &c, double q) {
  const bool wing = fabs(q) > (double)c.hfwid;
  QlgCoef vc = c.vcore;
  if (wing) {
    float a = 0.0f;
    if (q > h.qray) a = (float)(h.grad * (double)h_classical_wing(q));
    if (q > H_Q4000) {
      float xfac = 1.0f;
      if (q < 0.0) xfac = (float)((double)xfac + (double)0.13f * q / H_Q4000);
      a = a + xfac * c.resont + c.vdw;
    }
    vc = h_qlg_coef(a * c.idf);
  }
  float phi = 0.0f;
  for (int i = 0; i < h.io; i++) {
    const float vs = (float)((q - h.dq[i]) * (double)c.idf);
    const float xv = h_qlg_eval(tab, vc, vs) * c.idf;
    phi = (float)((double)phi + h.wt[i] * (double)xv);
  }
  if (wing && q > H_REDTHRESH) {
    if (q <= H_Q4000) {
      float x = (float)h_lyman_interp(H_LYH2, 91, 200.0f, -22000.0f, q * H_LYA0);
      phi = (float)((double)phi + H_LYA0 * (double)c.tothi * (double)powf(10.0f, x));
      x = (float)h_lyman_interp(H_LYH2PLUS, 111, 100.0f, -15000.0f, q * H_LYA0);
      phi = (float)((double)phi + H_LYA0 * (double)c.ne * (double)powf(10.0f, x));
      phi = (float)((double)phi + (double)0.5f * h_stark_eval(c.st, q));
    } else {
      double xstark = (double)0.5f * h_stark_eval(c.st, q);
      if (q < 0.0 && xstark > 0.0 && c.xholt4000 > 0.0) {
        const double sat4000 = H_LYA0 * (double)c.ne * pow(10.0, (double)(H_LYH2PLUS[110] - 14.0f));
        const float xfac = (float)(1.0 + (sat4000 / c.xholt4000 - 1.0) * q / H_Q4000);
        xstark = xstark * (1.0 + (double)xfac);
      }
      phi = (float)((double)phi + xstark);
    }
  }
  return phi;
}

__device__ __forceinline__ float h_profile(const float2 *tab, const HLineDev &h, const HCell &c, double q) {
  return c.lymanalf ? h_lyman_voigt(tab, h, c, q) : h_voigt(tab, h, c, q);
}

struct HCellsDev {
  const float *vproj, *inv_df, *temp, *ni, *ne, *tothi, *vbar2h, *fo, *t3nhe;
};

// hprofile at nq detunings per cell (the prepared cell of hcell_prepare), one warp
// per cell, lanes over q; phi (ncell, nq), q fastest
__global__ void k_h_profile(HLineDev h, const float2 *tab, long long ncell, HCellsDev cl, int nq, const double *q,
                            float *phi) {
  const int lane = threadIdx.x & 31;
  const long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= ncell) return;
  HCell hc;
  h_cell_prepare(h, cl.temp[c], cl.ne[c], cl.fo[c], cl.vbar2h[c], cl.tothi[c], cl.t3nhe[c], cl.inv_df[c], hc);
  for (int i = lane; i < nq; i += 32) phi[(size_t)c * nq + i] = h_profile(tab, h, hc, q[i]);
}

// add_h_opacities (hprofl_mod.f90:208-385), analytic profiles: one warp per cell.
// From f0 the profile is evaluated 32 frequencies at a time, upwards and then
// downwards, and added until (and including) the first point whose opacity falls
// below 1e-7 times the continuum at f0 -- the reference's walk, each point once.
__global__ void k_h_opacity(HLineDev h, const float2 *tab, double Bij, int f0, int nf, const double *nu,
                            long long ncell, HCellsDev cl, const float *bi, const float *bj, float *chi, float *eta,
                            const float *cont, int *used, unsigned *strength) {
  const int lane = threadIdx.x & 31;
  const long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= ncell) return;
  const float tol = 1e-7f;
  const float inv_nu0 = (float)(1.0 / h.nu0);
  const float idf = cl.inv_df[c];
  const float v = (float)((double)(cl.vproj[c] + 1.0f) * h.nu0);
  const float Rij = (float)((double)cl.ni[c] * Bij);
  const float cchi = bi ? Rij * bi[c] : Rij, ceta = bj ? Rij * bj[c] : Rij;
  HCell hc;
  h_cell_prepare(h, cl.temp[c], cl.ne[c], cl.fo[c], cl.vbar2h[c], cl.tothi[c], cl.t3nhe[c], idf, hc);
  const size_t base = (size_t)nf * (size_t)c;
  const float c0 = cont[base + f0];
  const float ref = tol * c0;
  if (!(ref >= ref)) return;   // a NaN reference: the reference's loops do not start
  for (int dir = 0; dir < 2; dir++) {
    for (int k = 0;; k += 32) {
      const int f = dir == 0 ? f0 + k + lane : f0 - 1 - k - lane;
      const bool in = dir == 0 ? f < nf : f >= 0;
      float lchi = 0.0f, leta = 0.0f;
      if (in) {
        const double q = (nu[f] - (double)v) * (double)inv_nu0;
        const float phi = h_profile(tab, h, hc, q);
        lchi = phi * cchi;
        leta = phi * ceta;
      }
      // the walk adds points while the previous one held lchi >= ref: up to and
      // including the first point below it, or the end of the grid
      const unsigned stop = __ballot_sync(0xffffffffu, !in || !(lchi >= ref));
      const int last = stop ? __ffs(stop) - 1 : 31;
      if (in && lane <= last) {
        chi[base + f] = chi[base + f] + lchi;
        eta[base + f] = eta[base + f] + leta;
        if (dir == 0 && k == 0 && lane == 0) {
          atomicOr(used, 1);
          const float s = lchi / c0;
          if (s > 0.0f) atomicMax(strength, __float_as_uint(s));
        }
      }
      if (stop) break;
    }
  }
}

}  // namespace m3d

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
#include <cfloat>

#include "m3d_htables.cuh"
#include "m3d_qlg.cuh"

namespace m3d {

struct HLineDev {
  int n, m, bpo, io;
  int opts, pad;
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

// ---- the tabulated profiles of HOP/hvcs_mod.f90 (VCS tables of Lemke 1997 or
// Stehle & Hutcheon 1999).  One series (Balmer, Paschen, Brackett) as read by
// read_vcs_grid, laid out as its grid_vcs(i, j, kk, l, k) with the wavelength
// fastest; the kernels read it from global memory, lanes along the wavelength.
constexpr int VCS_NW = 44, VCS_NT = 4, VCS_NE = 13, VCS_NH = 13, VCS_NL = 18;

struct VcsSeries {
  int loaded, nlines, radiative;
  int nlow[VCS_NL], nup[VCS_NL], nhhnr[VCS_NL];
  float grid[VCS_NL][VCS_NE][VCS_NT][VCS_NH][VCS_NW];
  float tslope[VCS_NL][VCS_NE][VCS_NT][VCS_NW];
  float nw[VCS_NW], nt[VCS_NT], ne[VCS_NE], nh[VCS_NH], dw_lin[VCS_NW], nw_invdx;
  double dw_first, dw_last;
};

// vcs_profile_t (hvcs_mod.f90:94-104) without its lp, which lives in shared memory
struct VcsCell {
  double lognorm, lam0, q_tail, ta, ts;
  int ok;
};

// what the host resolves for a line: its series and row, and the table's flags
struct VcsLine {
  const VcsSeries *ser;     // the line's series; ser1 the Balmer one, whose axis vcs_eval uses
  const VcsSeries *ser1;
  int use, row, resonance, radiative;
};

// pchip_slopes4 (interpol_mod.f90:193-235), the interior slope of node i (0-based)
__host__ __device__ __forceinline__ float vcs_pchip4_interior(const float *x, const float *y, int i, int ys) {
  const float dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
  const float dym = y[i * ys] - y[(i - 1) * ys], dyp = y[(i + 1) * ys] - y[i * ys];
  if (dym == 0 || dyp == 0) return 0.0f;
  const double d1 = (double)(dym / dxm), d2 = (double)(dyp / dxp);
  if (copysign(1.0, d1) != copysign(1.0, d2)) return 0.0f;
  const double alpha = (double)((1.0f + dxm / (dxp + dxm)) / 3.0f);
  return (float)(1.0 / ((1.0 - alpha) / d1 + alpha / d2));
}

// pchip_slopes4 over the window imin = j, imax = j + 1 of n >= 3 nodes (0-based j)
__device__ __forceinline__ void vcs_pchip4_pair(const float *x, const float *y, int ys, int n, int j, float &sj,
                                                float &sj1) {
  sj = j == 0 ? 2.0f * (y[ys] - y[0]) / (x[1] - x[0]) - vcs_pchip4_interior(x, y, 1, ys)
              : vcs_pchip4_interior(x, y, j, ys);
  sj1 = j + 1 == n - 1
            ? 2.0f * (y[(n - 1) * ys] - y[(n - 2) * ys]) / (x[n - 1] - x[n - 2]) - vcs_pchip4_interior(x, y, n - 2, ys)
            : vcs_pchip4_interior(x, y, j + 1, ys);
}

// hermite_value4 (interpol_mod.f90:125-140)
__device__ __forceinline__ float vcs_hermite4(float t, float h, float y0, float y1, float m0, float m1) {
  const float t2 = t * t, t3 = t2 * t;
  const float p = 3.0f * t2 - 2.0f * t3;
  return (1.0f - p) * y0 + p * y1 + h * (((t3 - 2.0f * t2) + t) * m0 + (t3 - t2) * m1);
}

// bracket (hvcs_mod.f90:508-520), 0-based
__device__ __forceinline__ int vcs_bracket(float x, const float *a, int n) {
  int j = 0;
  for (int kk = 0; kk < n - 1; kk++)
    if (x >= a[kk]) j = kk;
  return j;
}

// qpol (hvcs_mod.f90:431-466), for the short axes qpol4 hands it (1-based k as there)
__device__ __forceinline__ float vcs_qpol(float x, const float *a, const float *f, int fs, int no) {
  int k = no - 1;
  if (!(x > a[no - 1])) {
    k = 1;
    if (!(x < a[0] || no == 2)) {
      int nn = no;
      while (k != nn - 1) {
        const int i = (k + nn) / 2;
        if (a[i - 1] >= x) nn = i;
        else k = i;
      }
      if (k == no - 1) k = k - 1;
      const float u = x - a[k - 1], v = x - a[k], w = x - a[k + 1];
      const float fk = f[(k - 1) * fs], fk1 = f[k * fs], fk2 = f[(k + 1) * fs];
      const float y = (fk - fk1) / (v - u);
      const float z = (fk1 - fk2) / (w - v);
      if (y * z > 0.0f) return fk + u * y / (1.0f - v * (y - z) / (fk - fk2));
      return fk + u * (y + v * (y - z) / (w - u));
    }
  }
  return f[(k - 1) * fs] + (f[k * fs] - f[(k - 1) * fs]) * (x - a[k - 1]) / (a[k] - a[k - 1]);
}

// qpol4 (hvcs_mod.f90:528-554) on values at stride fs
__device__ __forceinline__ float vcs_qpol4(float x, const float *a, const float *f, int fs, int no) {
  if (no < 3) return vcs_qpol(x, a, f, fs, no);
  const int j = vcs_bracket(x, a, no);
  float sj, sj1;
  vcs_pchip4_pair(a, f, fs, no, j, sj, sj1);
  const float h = a[j + 1] - a[j];
  const float t = (x - a[j]) / h;
  return vcs_hermite4(t, h, f[j * fs], f[(j + 1) * fs], sj, sj1);
}

// qpol_w (hvcs_mod.f90:472-503) on the wavelength axis of series S
__device__ __forceinline__ float vcs_qpol_w(float x, const VcsSeries &S, const float *f) {
  const float *a = S.nw;
  int k;
  if (x > a[VCS_NW - 1]) {
    k = VCS_NW - 2;
    return f[k] + (f[k + 1] - f[k]) * (x - a[k]) / (a[k + 1] - a[k]);
  } else if (x < a[0]) {
    k = 0;
    return f[k] + (f[k + 1] - f[k]) * (x - a[k]) / (a[k + 1] - a[k]);
  }
  k = (int)((x - a[0]) * S.nw_invdx) + 1;
  k = k < 1 ? 1 : (k > VCS_NW - 2 ? VCS_NW - 2 : k);
  k -= 1;
  const float u = x - a[k], v = x - a[k + 1], w = x - a[k + 2];
  const float y = (f[k] - f[k + 1]) / (v - u);
  const float z = (f[k + 1] - f[k + 2]) / (w - v);
  if (y * z > 0.0f) return f[k] + u * y / (1.0f - v * (y - z) / (f[k] - f[k + 2]));
  return f[k] + u * (y + v * (y - z) / (w - u));
}

// vcs_prepare with vcs_cell_profile and tail_coef (hvcs_mod.f90:262-282, 319-327,
// 349-426) for one warp's cell: lanes build lp(i) over the wavelength nodes into
// lp (shared memory, 44 floats), then every lane forms the area in node order
__device__ __forceinline__ void vcs_prepare_warp(const VcsLine &L, double nu0, float temp, float ne, float nh,
                                                 float *lp, VcsCell &c) {
  const VcsSeries &S = *L.ser;
  const int r = L.row, nn = S.nhhnr[r];
  float tlog = log10f(fmaxf(temp, 1.0f));
  float nelog = log10f(fmaxf(ne, 1.0f));
  float nhlog = log10f(fmaxf(nh, 1.0f));
  if (nelog < S.ne[0]) nelog = S.ne[0];
  nelog = fminf(nelog, S.ne[VCS_NE - 1]);
  tlog = fminf(fmaxf(tlog, S.nt[0]), S.nt[VCS_NT - 1]);
  if (nn > 1) nhlog = fminf(fmaxf(nhlog, S.nh[0]), S.nh[nn - 1]);
  const int jt = vcs_bracket(tlog, S.nt, VCS_NT);
  const float ht = S.nt[jt + 1] - S.nt[jt];
  const float tt = (tlog - S.nt[jt]) / ht;
  const int je = vcs_bracket(nelog, S.ne, VCS_NE);
  const float he = S.ne[je + 1] - S.ne[je];
  const float te = (nelog - S.ne[je]) / he;
  const int le0 = je - 1 < 0 ? 0 : je - 1;
  const int le1 = je + 2 > VCS_NE - 1 ? VCS_NE - 1 : je + 2;
  const int ns = le1 - le0 + 1;
  for (int i = threadIdx.x & 31; i < VCS_NW; i += 32) {
    float ve[4];
    for (int l = le0; l <= le1; l++) {
      float v;
      if (nn > 1) {
        float vt[VCS_NT];
        for (int kk = 0; kk < VCS_NT; kk++) vt[kk] = vcs_qpol4(nhlog, S.nh, &S.grid[r][l][kk][0][i], VCS_NW, nn);
        v = vcs_qpol4(tlog, S.nt, vt, 1, VCS_NT);
      } else {
        v = vcs_hermite4(tt, ht, S.grid[r][l][jt][0][i], S.grid[r][l][jt + 1][0][i], S.tslope[r][l][jt][i],
                         S.tslope[r][l][jt + 1][i]);
      }
      ve[l - le0] = v;
    }
    float sj, sj1;
    vcs_pchip4_pair(S.ne + le0, ve, 1, ns, je - le0, sj, sj1);
    lp[i] = vcs_hermite4(te, he, ve[je - le0], ve[je - le0 + 1], sj, sj1);
  }
  __syncwarp();
  float plin = powf(10.0f, lp[0]);
  float area = plin * S.dw_lin[0];
  for (int i = 0; i < VCS_NW - 1; i++) {
    const float dl = S.dw_lin[i + 1] - S.dw_lin[i];
    const float plin_next = powf(10.0f, lp[i + 1]);
    area = area + 0.5f * (plin + plin_next) * dl;
    plin = plin_next;
  }
  area = 2.0f * area;
  const float lognorm = log10f(area);
  const VcsSeries &B = *L.ser1;
  c.ok = 1;
  c.lognorm = (double)lognorm;
  c.lam0 = (2.99792458e10 * 1.e8) / nu0;
  c.q_tail = B.dw_last / c.lam0;
  const double a = (double)B.nw[VCS_NW - 2];
  const double slope = (double)(lp[VCS_NW - 1] - lp[VCS_NW - 2]) / (double)(B.nw[VCS_NW - 1] - B.nw[VCS_NW - 2]);
  c.ts = slope;
  c.ta = 2.30258509299404568402 * ((double)lp[VCS_NW - 2] - slope * a - c.lognorm) + (1.0 + slope) * log(c.lam0);
}

// vcs_eval (hvcs_mod.f90:286-313)
__device__ __forceinline__ double vcs_eval(const VcsLine &L, const VcsCell &c, const float *lp, double q) {
  if (!c.ok) return 0.0;
  const double dlam = fabs(q) * c.lam0;
  const double deltaw = log10(fmax(dlam, L.ser1->dw_first));
  const double p = (double)vcs_qpol_w((float)deltaw, *L.ser1, lp);
  return exp(2.30258509299404568402 * (p - c.lognorm)) * c.lam0;
}

// vcs_tail (hvcs_mod.f90:333-343)
__device__ __forceinline__ double vcs_tail(const VcsCell &c, double lnq) { return c.ok ? exp(c.ta + c.ts * lnq) : 0.0; }

struct HCell {
  float idf, ne, tothi, resont, vdw, hwstk, hwlor, hfwid;
  float hwadd;
  int use_vcs;
  VcsCell vcs;
  const float *lp;     // the cell's table profile (shared memory), when use_vcs
  int lymanalf;
  HStark st;
  QlgCoef vcore, vwing, vwing_ray;
  double xholt4000;
};

// hcell_prepare (hprofl_mod.f90:388-438), the analytic branch
__device__ __forceinline__ void h_cell_prepare(const HLineDev &h, const VcsLine &L, float *lp, float temp, float ne,
                                               float fo, float vbar2h, float tothi, float t3nhe, float idf, HCell &c) {
  c.idf = idf;
  c.ne = ne;
  c.tothi = tothi;
  c.resont = (float)((double)tothi * h.gw1);
  if (h.gw2 != 0.0) c.resont = (float)((double)c.resont * pow((double)vbar2h, h.gw2));
  c.hwstk = (float)(h.gstk * (double)fo);
  c.vdw = (float)(h.gw3 * (double)t3nhe);
  c.hwlor = (float)(h.grad + (double)c.resont + (double)c.vdw);
  c.hfwid = fmaxf(fmaxf(1.0f / idf, c.hwlor), c.hwstk);
  c.hwadd = 0.0f;
  c.use_vcs = L.use;
  c.lp = lp;
  if (L.use) {
    // the tabulated profile, with the broadening the table lacks added as one
    // Lorentzian (hprofl_mod.f90:412-426)
    c.hwadd = c.vdw;
    if (!L.radiative) c.hwadd = c.hwadd + (float)h.grad;
    if (h.bpo || !L.resonance) c.hwadd = c.hwadd + c.resont;
    const float nh_table = (h.bpo || (h.opts & 4)) ? 0.0f : tothi;
    c.hfwid = fmaxf(1.0f / idf, c.hwadd);
    vcs_prepare_warp(L, h.nu0, temp, ne, nh_table, lp, c.vcs);
    c.lymanalf = 0;
    return;
  }
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

// added_wing (hprofl_mod.f90:560-574)
__device__ __forceinline__ float h_added_wing(const HCell &c, double d) {
  if (fabs(d) > (double)c.hfwid)
    return (float)((double)c.hwadd / (H_PI * (d * d + (double)c.hwadd * (double)c.hwadd))) * h_classical_wing(d);
  return 0.0f;
}

// vcs_fine (hprofl_mod.f90:514-536)
__device__ __forceinline__ float h_vcs_fine(const VcsLine &L, const HLineDev &h, const HCell &c, double q) {
  float phi;
  if (fabs(q) - h.dqmax > c.vcs.q_tail) {
    phi = (float)vcs_tail(c.vcs, log(fabs(q - h.dqbar)));
    if (c.hwadd > 0.0f) phi = phi + h_added_wing(c, q - h.dqbar);
    return phi;
  }
  phi = 0.0f;
  for (int i = 0; i < h.io; i++) phi = (float)((double)phi + h.wt[i] * (double)(float)vcs_eval(L, c.vcs, c.lp, q - h.dq[i]));
  if (c.hwadd > 0.0f)
    for (int i = 0; i < h.io; i++) phi = (float)((double)phi + h.wt[i] * (double)h_added_wing(c, q - h.dq[i]));
  return phi;
}

__device__ __forceinline__ float h_profile(const float2 *tab, const VcsLine &L, const HLineDev &h, const HCell &c,
                                           double q) {
  if (c.use_vcs) return h_vcs_fine(L, h, c, q);
  return c.lymanalf ? h_lyman_voigt(tab, h, c, q) : h_voigt(tab, h, c, q);
}

// profile_at (hprofl_mod.f90:336-350): past qt every component is on the table's
// power-law tail, from ln|d| of the rest-frame detuning and the cell's shift vp
__device__ __forceinline__ float h_profile_at(const float2 *tab, const VcsLine &L, const HLineDev &h, const HCell &c,
                                              double qt, double vp, double nu_f, double q) {
  if (fabs(q) > qt) {
    double d = (nu_f - h.nu0) / h.nu0 - h.dqbar;
    d = copysign(fmax(fabs(d), DBL_MIN), d);
    const double lnd = log(fabs(d)), invd = 1.0 / d;
    const double r = vp * invd;
    float phi = (float)vcs_tail(c.vcs, lnd - r * (1.0 + 0.5 * r));
    if (c.hwadd > 0.0f) phi = phi + h_added_wing(c, q - h.dqbar);
    return phi;
  }
  return h_profile(tab, L, h, c, q);
}

struct HCellsDev {
  const float *vproj, *inv_df, *temp, *ni, *ne, *tothi, *vbar2h, *fo, *t3nhe;
};

// hprofile at nq detunings per cell (the prepared cell of hcell_prepare), one warp
// per cell, lanes over q; phi (ncell, nq), q fastest
__global__ void __launch_bounds__(256) k_h_profile(HLineDev h, VcsLine L, const float2 *tab, long long ncell,
                                                    HCellsDev cl, int nq, const double *q, float *phi) {
  __shared__ float lps[8][VCS_NW];
  const int lane = threadIdx.x & 31;
  const long long c = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= ncell) return;
  HCell hc;
  h_cell_prepare(h, L, lps[threadIdx.x >> 5], cl.temp[c], cl.ne[c], cl.fo[c], cl.vbar2h[c], cl.tothi[c], cl.t3nhe[c],
                 cl.inv_df[c], hc);
  for (int i = lane; i < nq; i += 32) phi[(size_t)c * nq + i] = h_profile(tab, L, h, hc, q[i]);
}

// add_h_opacities (hprofl_mod.f90:208-385), analytic profiles: one warp per cell.
// From f0 the profile is evaluated 32 frequencies at a time, upwards and then
// downwards, and added until (and including) the first point whose opacity falls
// below 1e-7 times the continuum at f0 -- the reference's walk, each point once.
__global__ void __launch_bounds__(256) k_h_opacity(HLineDev h, VcsLine L, const float2 *tab, double Bij, int f0,
                                                    int nf, const double *nu, long long ncell, HCellsDev cl,
                                                    const float *bi, const float *bj, float *chi, float *eta,
                                                    const float *cont, int *used, unsigned *strength) {
  __shared__ float lps[8][VCS_NW];
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
  h_cell_prepare(h, L, lps[threadIdx.x >> 5], cl.temp[c], cl.ne[c], cl.fo[c], cl.vbar2h[c], cl.tothi[c], cl.t3nhe[c],
                 idf, hc);
  const double qt = hc.use_vcs ? hc.vcs.q_tail + h.dqmax : HUGE_VAL;
  const double vp = (double)cl.vproj[c];
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
        const float phi = h_profile_at(tab, L, h, hc, qt, vp, nu[f], q);
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

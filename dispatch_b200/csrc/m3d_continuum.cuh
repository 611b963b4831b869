// Continuum opacity of a window, HOP's composition_type%continuum_opacities
// (HOP/composition_mod.f90:2893-2984):
//   add_hrest                        :3807-3846
//   the absdat components            bftrans_mod.f90: absorption_factor :476-531,
//                                    interp_xkap :235-452 (their wavelength stencils,
//                                    load_lam_interp_weights :100-198, on the host)
//   components tabulated with stimulated emission, over 1 - beta   :2935-2970
//   boltzmann_factor                 :2822-2852
//   electron_scattering, rayleigh_scattering   :3851-3939
//   'H BF' under occupation probabilities: wcalc2   level_mod.f90:149-279 (its
//                                    per-wavelength set-up, calc_x_and_k :77-94, on the host)
// One warp per cell: the lanes first form each component's temperature stencil and
// absorption factor for the cell (one component per lane), then run along the
// window's wavelengths, each adding the components in their order.  Kinds follow the
// Fortran: tables, xhat and sigma real(4); the EOS state, the absorption factors and
// the wavelength cubes real(8); a real(4) value updated from a real(8) expression is
// rounded once where the Fortran assigns it.
#pragma once
#include "m3d_math.cuh"

namespace m3d {

constexpr int kContWarps = 4;     // warps (cells) per block
constexpr int kContMaxComp = 64;  // components of one call
constexpr int kContMaxRows = 1024;  // table rows a window reads, over all components (per cell, in shared memory)
constexpr int kContMaxTab = 8192;   // their table entries at every temperature node (per block, in shared memory)
constexpr int kContKF = 8;          // wavelengths a lane holds in one pass over the components

// wcalc2's per-wavelength set-up of an 'H BF' level (level_mod.f90:186-218): cls 0
// none, 1 beyond the series limit, 2 below it (a dissolved upper level); qcut =
// 2.0898E-26/(2 i^5) (real(4)) times the cut beyond the alpha line, the real(8) product
// g(f) starts from; x1, x2, kk = calc_x_and_k of the state, kd its kk in real(8)
struct OccFDev {
  double qcut, kd;
  float x1, x2, kk;
  int cls;
};

struct __align__(16) BfCompDev {
  int kind, istim, nnu, ntt, ilogl, lam3, log_table, kvadt, minet, maxet, iteta, k, fs, fe, active;
  // the table rows the window's stencils read (0-based r0 .. r0 + nrow - 1), their
  // place in the cell's shared row buffer and that of their entries at every
  // temperature node in the block's shared table (-1: read from global memory)
  int r0, nrow, soff, toff;
  double xkap_scale, mint, maxt, ion_xion, level_g, level_xion, awgt;
  const double *tt;
  const float *xkap;      // (nnu, ntt)
  // (nlam) the wavelength stencil: the first node, 0-based (-1 where none), as int
  // bits in x, and the three Lagrange weights in y, z, w
  const float4 *wt;
  const unsigned char *quad;
  const double *n, *n2, *part, *level_n;
  // an 'H BF' level under occupation probabilities: occ, its occupation probability
  // per cell and the per-wavelength set-up
  int occ;
  const double *level_w;
  const OccFDev *occf;
};

static_assert(sizeof(BfCompDev) % 16 == 0, "descriptors staged in shared memory ahead of the tables");

struct ContCellsDev {
  const double *temp, *teta, *e_kT, *pe, *dxi, *ne, *nHI, *partHI, *nHeI, *nH2, *shield;
  double HI_xion;
  int helium_scattering;
};

// the wavelength terms every cell shares, formed once per call (k_continuum_lam)
// with the operations the per-cell expressions use: lambda^3 in real(8) and its
// real(4) rounding, rayleigh_scattering's xr and its two polynomials, the
// helium term's (500/lambda)^4 times the cross section (0 without helium
// scattering)
struct ContLamDev {
  const double *cube, *xr, *rayh, *rayh2, *he;
  const float *l3;
};

// a component's state at one cell: the temperature stencil and the absorption factor
struct BfCellDev {
  float w0, w1, w2, fakt1;
  int it, in_bounds, quadratic, edge;
};

// absorption_factor of one cell times xkap_scale, capped at the real(4) maximum
__device__ __forceinline__ float cont_factor(const BfCompDev &c, const ContCellsDev &S, int x) {
  const double ekt = S.e_kT[x], pe = S.pe[x], dxi = S.dxi[x];
  double fk = DBL_MAX;
  switch (c.kind) {
    case 1: fk = c.n[x]; break;
    case 2: fk = c.n[x] * pe; break;
    case 3: {
      if (c.occ) break;   // absorption_factor leaves huge(1d0): interp_xkap does not use it
      int k5 = c.k * c.k;
      k5 = k5 * k5 * c.k;
      // the default-real literal over the integer 2 k^5: a real(4) quotient
      fk = (double)__fdiv_rn(2.0898e-26f, (float)(2 * k5)) * c.level_n[x];
      break;
    }
    case 4:
      fk = exp(-ekt * (c.ion_xion - dxi) - c.part[x]);
      fk = (double)2.0898e-26f / (2 * 13.598434 * ekt) * fk * c.n[x];
      break;
    case 5: fk = c.n[x] * c.n2[x]; break;
    case 6: fk = 1e-40 * c.n[x] * c.n2[x]; break;
    case 7: fk = pe * c.n[x]; break;
    case 8: fk = pe * c.n[x]; fk = (1e-40 / 1.602189e-12) * ekt * fk; break;
    case 9: fk = c.n[x] * c.awgt / 6.023e23; break;
    case 10:
      fk = c.level_g * exp(-ekt * c.level_xion - c.part[x]);
      fk = fk * c.n[x];
      break;
  }
  const double v = fk * c.xkap_scale;
  return (float)(v < (double)FLT_MAX ? v : (double)FLT_MAX);
}

// interp_xkap's temperature stencil of one cell (:303-345)
__device__ __forceinline__ BfCellDev cont_tstencil(const BfCompDev &c, double temp, double teta) {
  BfCellDev r;
  r.w0 = r.w1 = r.w2 = 0.0f;
  r.it = 0;
  r.quadratic = 0;
  r.edge = 0;
  bool inb = true;
  if (!c.minet) inb = inb && (temp > c.mint);
  if (!c.maxet) inb = inb && (temp < c.maxt);
  r.in_bounds = inb;
  if (!inb) return r;
  const double t = c.iteta ? teta : temp;
  const double *tt = c.tt;
  const int ntt = c.ntt;
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
    r.quadratic = c.kvadt;
  }
  if (r.quadratic) {
    const int i = (it + 2 <= ntt) ? it : it - 1;
    const double *t3 = tt + (i - 1);
    const double dt1 = 1. / ((t3[0] - t3[1]) * (t3[0] - t3[2]));
    const double dt2 = 1. / ((t3[1] - t3[0]) * (t3[1] - t3[2]));
    const double dt3 = 1. / ((t3[2] - t3[0]) * (t3[2] - t3[1]));
    const double d1 = t - t3[0], d2 = t - t3[1], d3 = t - t3[2];
    r.w0 = (float)(d2 * d3 * dt1);
    r.w1 = (float)(d1 * d3 * dt2);
    r.w2 = (float)(d1 * d2 * dt3);
    r.it = i;
  } else {
    const double dtdt1 = 1. / (tt[it] - tt[it - 1]);
    r.w0 = (float)((t - tt[it - 1]) * dtdt1);
    r.it = it;
  }
  return r;
}

// row j (1-based) of the table at the cell's temperature, converted to the form of
// the wavelength interpolation (:332-357)
__device__ __forceinline__ float cont_row(const BfCompDev &c, const BfCellDev &r, int j) {
  const float *tab = c.xkap + (j - 1);
  const size_t nnu = (size_t)c.nnu;
  float y;
  if (r.quadratic) {
    const size_t i = (size_t)r.it;
    y = __fadd_rn(__fadd_rn(__fmul_rn(tab[nnu * (i - 1)], r.w0), __fmul_rn(tab[nnu * i], r.w1)),
                  __fmul_rn(tab[nnu * (i + 1)], r.w2));
  } else {
    const size_t it = (size_t)r.it;
    const float a = tab[nnu * (it - 1)], b = tab[nnu * it];
    y = __fadd_rn(__fmul_rn(__fsub_rn(b, a), r.w0), a);
    if (r.edge == 1) y = fminf(y, tab[0]);
    else if (r.edge == 2) y = fminf(y, tab[nnu * (c.ntt - 1)]);
  }
  if (c.log_table && !c.ilogl) y = exp4(y);
  else if (c.ilogl && !c.log_table) y = logf(fmaxf(y, FLT_MIN));
  return y;
}

// the same row from the block's staged table: entry (row, node) at
// stab[toff + node nrow + row - r0]
__device__ __forceinline__ float cont_row_s(const BfCompDev &c, const BfCellDev &r, const float *stab, int j) {
  const float *tab = stab + c.toff + (j - 1 - c.r0);
  const size_t nr = (size_t)c.nrow;
  float y;
  if (r.quadratic) {
    const size_t i = (size_t)r.it;
    y = __fadd_rn(__fadd_rn(__fmul_rn(tab[nr * (i - 1)], r.w0), __fmul_rn(tab[nr * i], r.w1)),
                  __fmul_rn(tab[nr * (i + 1)], r.w2));
  } else {
    const size_t it = (size_t)r.it;
    const float a = tab[nr * (it - 1)], b = tab[nr * it];
    y = __fadd_rn(__fmul_rn(__fsub_rn(b, a), r.w0), a);
    if (r.edge == 1) y = fminf(y, tab[0]);
    else if (r.edge == 2) y = fminf(y, tab[nr * (c.ntt - 1)]);
  }
  if (c.log_table && !c.ilogl) y = exp4(y);
  else if (c.ilogl && !c.log_table) y = logf(fmaxf(y, FLT_MIN));
  return y;
}

// one component's contributions at the lane's wavelengths f0 + 32 k (interp_xkap
// :358-385 and :386-426), each added to v[k] where the component reaches f; l3[f]
// is real(lambda^3).  The component's fields are read once for all of them.
template <int KF>
__device__ __forceinline__ void cont_comp(const BfCompDev &c, const BfCellDev &r, const float *rows, int f0,
                                          const float *__restrict__ l3, const ContCellsDev &S, int x,
                                          float (&v)[KF]) {
  if (!c.active) return;
  const int fs = c.fs, fe = c.fe, nnu = c.nnu, ilogl = c.ilogl, lam3 = c.lam3;
  const float4 *wt = c.wt;
  if (c.ntt > 1) {
    if (!r.in_bounds) return;
    const float fakt1 = r.fakt1;
    const int soff = c.soff;
    const float *yy = rows + soff - c.r0;   // yy[row], 0-based table rows
#pragma unroll
    for (int k = 0; k < KF; k++) {
      const int f = f0 + 32 * k;
      if (f < fs || f > fe) continue;
      const float4 w = __ldg(wt + f);
      const int iw = __float_as_int(w.x);
      float ab;
      if (iw >= 0) {
        float y1, y2, y3;
        if (soff >= 0) {
          y1 = yy[iw];
          y2 = yy[iw + 1];
          y3 = yy[iw + 3 < nnu ? iw + 2 : nnu - 1];
        } else {
          const int i = iw + 1;
          y1 = cont_row(c, r, i);
          y2 = cont_row(c, r, i + 1);
          y3 = cont_row(c, r, i + 2 < nnu ? i + 2 : nnu);
        }
        ab = __fadd_rn(__fadd_rn(__fmul_rn(y1, w.y), __fmul_rn(y2, w.z)), __fmul_rn(y3, w.w));
      } else {
        ab = ilogl ? -FLT_MAX : 0.0f;
      }
      if (ilogl) ab = exp4(ab);
      if (lam3) ab = __fmul_rn(ab, __ldg(l3 + f));
      v[k] = __fadd_rn(v[k], __fmul_rn(fakt1, ab));
    }
  } else if (c.occ) {
    // interp_xkap_2's table at the window, then wcalc2 for the cell (bftrans_mod.f90
    // :398-428, level_mod.f90:220-277): w, 1 - w, the level's population and
    // 4 pi/3 n_H of the cell are in r; shield, ne and 4 pi/3 n_He are the cell's
    const float w = r.w0, omw = r.w1, n = r.w2, nh43 = r.fakt1;
    const double xd = S.shield[x];
    const float xs = (float)xd, ne1 = (float)S.ne[x], nhe43 = (float)(4.18879 * S.nHeI[x]);
    const float *xk = c.xkap;
    const unsigned char *quad = c.quad;
    const OccFDev *occf = c.occf;
    const float scale = (float)c.xkap_scale;
#pragma unroll
    for (int k = 0; k < KF; k++) {
      const int f = f0 + 32 * k;
      if (f < fs || f > fe) continue;
      const OccFDev o = occf[f];
      if (o.cls == 0) continue;
      const float4 wv = __ldg(wt + f);
      const int iw = __float_as_int(wv.x);
      float ab;
      if (iw < 0) {
        ab = 0.0f;
      } else {
        const float *yy = xk + iw;
        ab = __fadd_rn(0.0f, __fmul_rn(yy[0], wv.y));
        ab = __fadd_rn(ab, __fmul_rn(yy[1], wv.z));
        if (quad[f]) ab = __fadd_rn(ab, __fmul_rn(yy[2], wv.w));
        if (ilogl) ab = expf(ab);
      }
      if (lam3) ab = __fmul_rn(ab, __ldg(l3 + f));
      // g = real(2.0898E-26/(2 i^5) * cutfac * ab, 4), ab times real(xkap_scale, 4)
      const float g = (float)(o.qcut * (double)__fmul_rn(ab, scale));
      float d;
      if (o.cls == 1) {
        d = w;
      } else {
        // neutral perturbers E = exp(-a); charged ones C = frac/(1+frac), tested on
        // the real(8) product; w - wstar formed as (1 - wstar) - (1 - w) near w = 1
        const float a = __fadd_rn(__fmul_rn(nh43, o.x1), __fmul_rn(nhe43, o.x2));
        float E, omE;
        exp_neg0(a, E, omE);
        const float k1 = o.kk;
        const float xkk = __fmul_rn(xs, k1);
        float C = 1.0f, omC = 0.0f;
        if (xd * o.kd < 1e4) {
          const float den = __fadd_rn(1.0f, __fmul_rn(0.1285f, xkk));
          const float frac = __fdiv_rn(__fmul_rn(__fmul_rn(0.1402f, xkk), k1), __fmul_rn(ne1, den));
          C = __fdiv_rn(frac, __fadd_rn(1.0f, frac));
          omC = __fdiv_rn(1.0f, __fadd_rn(1.0f, frac));
        }
        d = (w > 0.5f) ? __fsub_rn(__fadd_rn(omE, __fmul_rn(E, omC)), omw) : __fsub_rn(w, __fmul_rn(E, C));
      }
      v[k] = __fadd_rn(v[k], __fmul_rn(__fmul_rn(d, n), g));
    }
  } else {
    const float fakt1 = r.fakt1;
    const float *xk = c.xkap;
    const unsigned char *quad = c.quad;
#pragma unroll
    for (int k = 0; k < KF; k++) {
      const int f = f0 + 32 * k;
      if (f < fs || f > fe) continue;
      const float4 w = __ldg(wt + f);
      const int iw = __float_as_int(w.x);
      float ab;
      if (iw < 0) {
        ab = 0.0f;
      } else {
        const float *yy = xk + iw;
        ab = __fadd_rn(0.0f, __fmul_rn(yy[0], w.y));
        ab = __fadd_rn(ab, __fmul_rn(yy[1], w.z));
        if (quad[f]) ab = __fadd_rn(ab, __fmul_rn(yy[2], w.w));
        if (ilogl) ab = expf(ab);
      }
      if (lam3) ab = __fmul_rn(ab, __ldg(l3 + f));
      v[k] = __fadd_rn(v[k], __fmul_rn(ab, fakt1));
    }
  }
}

// thomson = 8./3.*PI*(EC**2/(EM*CC**2))**2 (composition_mod.f90:3856), a real(8)
// parameter whose 8./3. is a default-real quotient
__device__ __forceinline__ double cont_thomson() {
  const double rq = (4.80325e-10 * 4.80325e-10) / (9.109534e-28 * (2.99792458e10 * 2.99792458e10));
  return (double)(8.0f / 3.0f) * 3.14159265359 * (rq * rq);
}

// the shared wavelength terms: rayleigh_scattering's per-wavelength xray2 and HeIscat
// (composition_mod.f90:3903-3911) and the H I and H2 polynomials in xr it forms per cell
__global__ void k_continuum_lam(int nlam, const double *__restrict__ lam, int helium, double *__restrict__ cube,
                                float *__restrict__ l3, double *__restrict__ xr_o, double *__restrict__ rayh_o,
                                double *__restrict__ rayh2_o, double *__restrict__ he_o) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nlam) return;
  const double l = lam[f];
  const double c3 = l * l * l;
  cube[f] = c3;
  l3[f] = (float)c3;
  double xr = 0.0;
  if (l > 1400.0) {
    const double m = l > 1026.0 ? l : 1026.0;
    xr = 1 / (m * m);
  }
  xr_o[f] = xr;
  rayh_o[f] = (double)5.799e-13f + xr * ((double)1.422e-6f + xr * (double)2.784f);
  rayh2_o[f] = (double)8.14e-13f + xr * ((double)1.28e-6f + xr * (double)1.61f);
  double he = 0.0;
  if (helium) {
    const double q = (double)500.f / l;
    const double q2 = q * q;
    he = (double)(0.66520e-24f * 4.f) * (q2 * q2);
  }
  he_o[f] = he;
}

// eight blocks per SM (64 registers): the latency of the stencil loads is hidden by
// occupancy, measured faster than 80 registers at six blocks and than 56 or 48 at
// nine or ten
__global__ void __launch_bounds__(kContWarps * 32, 8)
k_continuum(int ncomp, const BfCompDev *__restrict__ comps_g, int any_istim, int nlam, ContLamDev LW,
            const double *__restrict__ nu, int ncell, ContCellsDev S, const float *__restrict__ beta,
            float *__restrict__ xhat, float *__restrict__ sigma, int rows_used, int tab_used) {
  __shared__ BfCellDev sc[kContWarps][kContMaxComp];
  extern __shared__ __align__(16) float cont_sh[];
  BfCompDev *scomp = reinterpret_cast<BfCompDev *>(cont_sh);   // (ncomp) the components' descriptors
  float *cont_dyn = cont_sh + ncomp * (sizeof(BfCompDev) / sizeof(float));
  float *stab = cont_dyn;                                        // (tab_used) the staged table entries
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  BfCellDev *st = sc[wib];
  float *rows = cont_dyn + tab_used + (size_t)wib * rows_used;   // (rows_used) this cell's rows
  {
    const int nw = ncomp * (int)(sizeof(BfCompDev) / sizeof(int));
    const int *src = reinterpret_cast<const int *>(comps_g);
    int *dst = reinterpret_cast<int *>(scomp);
    for (int q = threadIdx.x; q < nw; q += blockDim.x) dst[q] = src[q];
  }
  __syncthreads();
  const BfCompDev *comps = scomp;
  // the window's table rows at every temperature node, once per block
  for (int j = 0; j < ncomp; j++) {
    const BfCompDev &c = comps[j];
    if (c.toff < 0) continue;
    const int m = c.nrow * c.ntt;
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
      const int node = q / c.nrow, row = q - node * c.nrow;
      stab[c.toff + q] = c.xkap[(size_t)(c.r0 + row) + (size_t)c.nnu * node];
    }
  }
  __syncthreads();
  const int nwarp = gridDim.x * kContWarps;
  const double thomson = cont_thomson();
  for (int x = blockIdx.x * kContWarps + wib; x < ncell; x += nwarp) {
    const double temp = S.temp[x], teta = S.teta[x];
    for (int j = lane; j < ncomp; j += 32) {
      const BfCompDev &c = comps[j];
      BfCellDev r;
      if (c.ntt > 1) {
        r = cont_tstencil(c, temp, teta);
      } else {
        r.w0 = r.w1 = r.w2 = 0.0f;
        r.it = 0;
        r.in_bounds = 1;
        r.quadratic = 0;
        r.edge = 0;
      }
      if (c.occ && c.ntt == 1) {
        // wcalc2's per-cell terms (level_mod.f90:222-229)
        const double wo = c.active ? c.level_w[x] : 0.0;
        r.w0 = (float)wo;
        r.w1 = (float)(1.0 - wo);
        r.w2 = c.active ? (float)c.level_n[x] : 0.0f;
        r.fakt1 = c.active ? (float)(4.18879 * c.n[x]) : 0.0f;
      } else {
        r.fakt1 = (c.active && r.in_bounds) ? cont_factor(c, S, x) : 0.0f;
      }
      st[j] = r;
    }
    __syncwarp();
    // the table rows at the cell's temperature, each formed once (interp_xkap's yy)
    for (int j = 0; j < ncomp; j++) {
      const BfCompDev &c = comps[j];
      if (c.soff < 0 || !c.active || !st[j].in_bounds) continue;
      for (int q = lane; q < c.nrow; q += 32) rows[c.soff + q] = cont_row_s(c, st[j], stab, c.r0 + q + 1);
    }
    __syncwarp();
    // add_hrest: the H I levels above n = 15, up to the lowered ionisation limit
    const double ekt = S.e_kT[x], dxi = S.dxi[x];
    const double nniv2 = (double)(15.5f * 15.5f);
    bool hrest_on = false;
    double hrest = 0.0;
    if (S.nHI && 13.598434 >= nniv2 * dxi) {
      double fakt = exp(-ekt * (S.HI_xion - dxi) - S.partHI[x]);
      fakt = (double)2.0898e-26f / (2 * 13.598434 * ekt) * fakt * S.nHI[x];
      hrest = exp(ekt * (13.598434 / nniv2 - dxi));
      hrest = fakt * (hrest - 1);
      hrest_on = true;
    }
    const double hk_T = (6.626176e-27 / 1.380662e-16) / temp;
    const double nHIr = S.nHI ? S.nHI[x] : 0.0, nHE = S.nHeI ? S.nHeI[x] : 0.0, nH2 = S.nH2 ? S.nH2[x] : 0.0;
    const double els = sigma ? thomson * S.ne[x] : 0.0;
    for (int f0 = lane; f0 - lane < nlam; f0 += 32 * kContKF) {
      float v[kContKF];
#pragma unroll
      for (int k = 0; k < kContKF; k++) {
        const int f = f0 + 32 * k;
        v[k] = (hrest_on && f < nlam) ? (float)((double)0.0f + hrest * __ldg(LW.cube + f)) : 0.0f;
      }
      for (int j = 0; j < ncomp; j++) {
        const BfCompDev &c = comps[j];
        if (!c.istim) cont_comp<kContKF>(c, st[j], rows, f0, LW.l3, S, x, v);
      }
      if (any_istim) {
        float tmp[kContKF];
#pragma unroll
        for (int k = 0; k < kContKF; k++) tmp[k] = 0.0f;
        for (int j = 0; j < ncomp; j++) {
          const BfCompDev &c = comps[j];
          if (c.istim) cont_comp<kContKF>(c, st[j], rows, f0, LW.l3, S, x, tmp);
        }
#pragma unroll
        for (int k = 0; k < kContKF; k++) {
          const int f = f0 + 32 * k;
          if (f >= nlam) break;
          float b;
          if (beta) {
            b = beta[(size_t)f + (size_t)nlam * x];
          } else {
            b = (float)exp(-nu[f] * hk_T);
            b = b > FLT_MIN ? b : FLT_MIN;
          }
          v[k] = __fadd_rn(v[k], __fdiv_rn(tmp[k], __fsub_rn(1.0f, b)));
        }
      }
#pragma unroll
      for (int k = 0; k < kContKF; k++) {
        const int f = f0 + 32 * k;
        if (f >= nlam) break;
        const size_t o = (size_t)f + (size_t)nlam * x;
        xhat[o] = v[k];
        if (sigma) {
          float s = (float)(0.0 + els);
          const double xr = __ldg(LW.xr + f);
          if (xr > 0.) {
            const double rayh = __ldg(LW.rayh + f) * nHIr;
            const double rayh2 = __ldg(LW.rayh2 + f) * nH2;
            s = (float)((double)s + (rayh + rayh2) * xr * xr);
          }
          sigma[o] = (float)((double)s + __ldg(LW.he + f) * nHE);
        }
      }
    }
    __syncwarp();
  }
}

// calc_x_and_k (level_mod.f90:77-94) in real(8), as the host forms it for wcalc2
__device__ __forceinline__ void h_calc_x_and_k(double ns, double &x1, double &x2, double &k) {
  const double rbohr = 5.29177349e-9;
  const double ns2 = ns * ns;
  const double rih = ns * sqrt(2.5 * ns2 + 0.5);
  const double t1 = rbohr * (rih + (double)1.73f), t2 = rbohr * (rih + (double)1.02f);
  x1 = t1 * t1 * t1;
  x2 = t2 * t2 * t2;
  double kk = (double)8.3e14f / (ns2 * ns2);
  if (ns > 3.) kk = kk * (double)5.33333333f * ns / ((ns + 1.0) * (ns + 1.0));
  k = kk * sqrt(kk);
}

// init_H_levels with compute_shield (composition_mod.f90:2604-2613, 2708-2768), one
// thread per cell: the shielding (1 + 0.08989 ne^0.16667/sqrt(T))^3.15/ne; the
// hydrogenic levels i = 1..nk, xion = Ryd (1 - 1/i^2) (a real(4) bracket), g = 2 i^2,
// n_i = g exp(-e_kT xion); with occupation probabilities w_i = wcalc (level_mod.f90:
// 108-142) and the partition function 1 / sum w_i n_i, else exp(-ln U) with the levels
// above n = sqrt(Ryd/dxi) dissolved where the first cell's dxi > 0 (the reference tests
// dxi(1,1,1)); then n_i = nHI n_i part
__global__ void k_h_levels(int ncell, int nk, int occupation, int dissolve, const double *__restrict__ temp,
                           const double *__restrict__ e_kT, const double *__restrict__ ne,
                           const double *__restrict__ dxi, const double *__restrict__ nHI,
                           const double *__restrict__ nHeI, const double *__restrict__ partHI,
                           double *__restrict__ shield, double *__restrict__ level_n, double *__restrict__ level_w) {
  const double ryd = 13.598434, pi43 = 4.18879;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const double nec = ne[c];
    double sh = (double)0.08989f * pow(nec, 0.16667) / sqrt(temp[c]);
    sh = pow(1.0 + sh, 3.15) / nec;
    shield[c] = sh;
    const double ekt = e_kT[c];
    double part = 0.0;
    if (occupation) {
      const double nh = nHI[c], nhe = nHeI[c];
      for (int i = 1; i <= nk; i++) {
        const float xi = 1.0f - 1.0f / (float)(i * i);
        const double n = (double)(2 * i * i) * exp(-ekt * (ryd * (double)xi));
        double x1, x2, k1;
        h_calc_x_and_k((double)i, x1, x2, k1);
        const double k2 = k1 * k1;
        double res = exp(-(pi43 * (nh * x1 + nhe * x2)));
        if (k1 * sh < 1e4) {
          const double frac = 0.1402 * sh * k2 / (nec * (1.0 + (double)0.1285f * sh * k1));
          res = res * (frac / (1.0 + frac));
        }
        level_w[c + (size_t)ncell * (i - 1)] = res;
        level_n[c + (size_t)ncell * (i - 1)] = n;
        part = part + res * n;
      }
      part = 1.0 / part;
    } else {
      part = exp(-partHI[c]);
      // a cell without lowering (dxi <= 0) keeps every level (int(sqrt(Ryd/0)) is
      // undefined in the reference)
      const bool cut = dissolve && dxi[c] > 0.0;
      const double h1 = cut ? sqrt(ryd / dxi[c]) : 0.0;
      const int nniv = cut && h1 < 2147483647.0 ? (int)h1 : 2147483647;
      for (int i = 1; i <= nk; i++) {
        const float xi = 1.0f - 1.0f / (float)(i * i);
        double n = (double)(2 * i * i) * exp(-ekt * (ryd * (double)xi));
        if (cut) {
          if (nniv < i) n = 0.0;
          else if (nniv == i) n = n * (h1 - (double)nniv);
        }
        level_n[c + (size_t)ncell * (i - 1)] = n;
      }
    }
    const double nh = nHI[c];
    for (int i = 1; i <= nk; i++) {
      double &n = level_n[c + (size_t)ncell * (i - 1)];
      n = nh * n * part;
    }
  }
}

}  // namespace m3d

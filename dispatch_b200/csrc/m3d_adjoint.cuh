// Reverse mode of the LTE synthesis pass (one window, every ray): the gradients of a
// loss L(flux) with respect to the pass's inputs, by a hand-written adjoint of each
// stage, run backwards:
//
//   flux <- ie <- I_top                  linear (save_intensity, rt_patch_mod.f90:4151-4208)
//   I_top <- rotated planes              k_quad_rot_column_adj: the fused sweep
//                                        (rotate_array + long_char_quadratic over all
//                                        slabs, rt_solvers_mod.f90:891-1020) reversed
//                                        column by column; the forward intensities are
//                                        checkpointed at the slab faces only and each
//                                        slab is recomputed from its face as it is
//                                        reversed
//   rotated planes <- chi, S             k_unrotate_adj: the transpose of the bilinear
//                                        shift of rotate_array (rt_patch_mod.f90:3809-
//                                        3866), a gather over the four columns that
//                                        tapped a cell, plus the PCHIP ghost's terms
//   chi, S <- chi_l, T, chi_c            k_units_adj: work_to_transfer_units and the
//                                        LTE background (rt_patch_mod.f90:2004-2023,
//                                        3518-3536, 3571-3651)
//   chi_l <- lnbase, e_kT, inv_df, gpref k_opacity_adj: add_opacity_equi's line loop
//                                        (linelist_mod.f90:729-960) replayed with the
//                                        forward's decisions, every deposited profile
//                                        point adding its sensitivities
//
// Non-differentiable decisions (line windows, the tolerance tests, the limiter
// branches, clamps) are taken as the forward takes them and held fixed.  QLG-bot's
// profile snaps to the nearest table node, which is piecewise constant in the
// abscissa; its derivative is taken from the continuous member the table samples:
// G(u) = 2^-u exactly, W(u) from the table's central differences.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "m3d_pipeline.cuh"

namespace m3d {

// minmod of the limited slopes as the quadratic solver forms it,
// m = (sgn a + sgn b) min(|a|, |b|, |a + b|/4), with its partial derivatives
template <typename T>
__device__ __forceinline__ void minmod_d(T a, T b, T &m, T &da, T &db) {
  const T h = (T)0.5 * (a + b);
  const T aa = tabs(a), ab = tabs(b), ah = tabs((T)0.5 * h);
  m = (tcopysign((T)1, a) + tcopysign((T)1, b)) * tmin(tmin(aa, ab), ah);
  if (tcopysign((T)1, a) != tcopysign((T)1, b)) { da = 0; db = 0; return; }
  if (ah <= aa && ah <= ab) { da = (T)0.5; db = (T)0.5; }
  else if (aa <= ab) { da = 2; db = 0; }
  else { da = 0; db = 2; }
}

// dq/dt of the parabolic moment q(t) = t - 2 U1/t = t - 2 + 2 U0/t:
// 1 - 2 (U0 - t E)/t^2, by its series below |t| = 1/2, where the closed form cancels
template <typename T>
__device__ __forceinline__ T dq_dt(T t, T E, T U0) {
  if (tabs(t) < (T)0.5) {
    // 2(U0 - tE)/t^2 = sum_{n>=2} (-1)^n 2(n-1)/n! t^(n-2)
    T p = (T)(-1.0 / 22680.0);
    p = fma_t(t, p, (T)(1.0 / 2880.0));
    p = fma_t(t, p, (T)(-1.0 / 420.0));
    p = fma_t(t, p, (T)(1.0 / 72.0));
    p = fma_t(t, p, (T)(-1.0 / 15.0));
    p = fma_t(t, p, (T)0.25);
    p = fma_t(t, p, (T)(-2.0 / 3.0));
    return -t * p;   // 1 - (1 + t p) = -t p
  }
  return (T)1 - (T)2 * (U0 - t * E) / (t * t);
}

template <typename T>
struct QStepGrad { T xu, xc, xd, su, sc, sd, Iu; };

// The adjoint of one quad_step: with gI = dL/dI_out, adds dL/d(each input) into g
template <typename T>
__device__ __forceinline__ void quad_step_adj(T xu, T xc, T xd, T su, T sc, T sd, T Iu, bool at_target, T rdsup,
                                              T dsup1, T dsup2, T dtmax, T Imax, T gI, QStepGrad<T> &g) {
  const T dtmin = (T)1e-20f;
  // forward, with the branch choices
  const T t1 = (xc - xu) * rdsup, t3 = (xd - xc) * rdsup;
  T t2, d21, d23;
  minmod_d(t1, t3, t2, d21, d23);
  const T dtup_r = fma_t(dsup2, t1 - t2, dsup1 * (xu + xc));
  const T dtdn_r = fma_t(dsup2, t2 - t3, dsup1 * (xd + xc));
  const T dtup = tmax(tcopysign(tmax(tabs(dtup_r), dtmin), dtup_r), dtmax);
  const T dtdn = tmax(tcopysign(tmax(tabs(dtdn_r), dtmin), dtdn_r), dtmax);
  const bool up_free = tabs(dtup_r) >= dtmin && dtup_r > dtmax;
  const bool dn_free = tabs(dtdn_r) >= dtmin && dtdn_r > dtmax;
  const T dt = at_target ? dtup : dtdn;
  const T rdt = (T)1 / dt;
  T ex, U0, U1, q;
  parab_moments(dt, ex, U0, U1, q);
  T s1, s3;
  if (at_target) { s1 = (sc - su) * rdt; s3 = (sd - sc) / dtdn; }
  else { s1 = (sc - su) / dtup; s3 = (sd - sc) * rdt; }
  T ds, dd1, dd3;
  minmod_d(s1, s3, ds, dd1, dd3);
  T A, B, C, I;
  if (at_target) {
    B = ((T)2 * U1 - q) * rdt; A = U0 - B; C = q - U1;
    I = fma_t(C, ds, fma_t(B, sc, fma_t(A, su, Iu * ex)));
  } else {
    A = q * rdt; B = U0 - A; C = U1 - q;
    I = fma_t(C, ds, fma_t(B, sc, fma_t(A, sd, Iu * ex)));
  }
  if (tabs(I) > Imax) return;   // clamped: no sensitivity
  // backward
  g.Iu += gI * ex;
  const T g_ex = gI * Iu, g_C = gI * ds, g_ds = gI * C;
  T g_U0, g_U1, g_q, g_rdt, g_dtup = 0, g_dtdn = 0;
  if (at_target) {
    const T g_A = gI * su, g_B = gI * sc;
    g.su += gI * A;
    g.sc += gI * B;
    const T g_Bt = g_B - g_A;
    g_U0 = g_A;
    g_q = g_C - g_Bt * rdt;
    g_U1 = -g_C + (T)2 * g_Bt * rdt;
    g_rdt = g_Bt * ((T)2 * U1 - q);
  } else {
    const T g_A = gI * sd, g_B = gI * sc;
    g.sd += gI * A;
    g.sc += gI * B;
    const T g_At = g_A - g_B;
    g_U0 = g_B;
    g_U1 = g_C;
    g_q = -g_C + g_At * rdt;
    g_rdt = g_At * q;
  }
  const T g_s1 = g_ds * dd1, g_s3 = g_ds * dd3;
  if (at_target) {
    g.sc += g_s1 * rdt; g.su -= g_s1 * rdt; g_rdt += g_s1 * (sc - su);
    g.sd += g_s3 / dtdn; g.sc -= g_s3 / dtdn; g_dtdn -= g_s3 * s3 / dtdn;
  } else {
    g.sc += g_s1 / dtup; g.su -= g_s1 / dtup; g_dtup -= g_s1 * s1 / dtup;
    g.sd += g_s3 * rdt; g.sc -= g_s3 * rdt; g_rdt += g_s3 * (sd - sc);
  }
  const T g_dt = -g_rdt * rdt * rdt - g_ex * ex + g_U0 * ex + g_U1 * U0 + g_q * dq_dt(dt, ex, U0);
  if (at_target) g_dtup += g_dt; else g_dtdn += g_dt;
  const T gu = up_free ? g_dtup : (T)0, gd = dn_free ? g_dtdn : (T)0;
  T g_t1 = dsup2 * gu, g_t3 = -dsup2 * gd;
  const T g_t2 = -dsup2 * gu + dsup2 * gd;
  g.xu += dsup1 * gu;
  g.xc += dsup1 * (gu + gd);
  g.xd += dsup1 * gd;
  g_t1 += g_t2 * d21;
  g_t3 += g_t2 * d23;
  g.xc += (g_t1 - g_t3) * rdsup;
  g.xu -= g_t1 * rdsup;
  g.xd += g_t3 * rdsup;
}

// One step forward (for the recomputation inside a slab)
template <typename T>
__device__ __forceinline__ T quad_fwd(T xu, T xc, T xd, T su, T sc, T sd, T Iu, bool at_target, const QuadConst &qc,
                                      T dtmax, T Imax) {
  T I, pl;
  quad_step<T>(xu, xc, xd, su, sc, sd, Iu, at_target, (T)qc.rdsup, (T)qc.dsup1, (T)qc.dsup2, dtmax, Imax, false, I,
               pl);
  return I;
}

// pchip ghost value and its partials in the two unrotated planes
__device__ __forceinline__ float pchip_ghost_d(float y1, float y2, const PchipConst &pc, float &d1, float &d2) {
  const float v = pchip_ghost(y1, y2, pc);
  const float raw = (pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * ((2.0f * (y2 - y1)) / pc.dx1 - 0.0f) + pc.cm1 * 0.0f);
  const bool live = raw > 0.0f;
  d1 = live ? pc.c0 - 2.0f * pc.cm0 : 0.0f;
  d2 = live ? pc.p + 2.0f * pc.cm0 : 0.0f;
  return v;
}

constexpr int ADJ_MAXN = 64;     // planes per slab the reverse sweep holds per thread
constexpr int ADJ_MAXSLAB = 64;  // slabs per column

__device__ __forceinline__ void rot_at(const float *chi, const float *S, size_t plane, int z, const RotCol &r, int f,
                                       int x, int y, int nf, int nx, int ny, float &xv, float &sv) {
  const Taps t = load_taps(chi, S, plane * z, r, f, x, y, nf, nx, ny);
  combine(t, r, xv, sv);
}

// The reverse of k_quad_rot_column for one ray.  g_top: dL/dI_top (nf, nx, ny).
// Outputs dL/d(rotated chi) and dL/d(rotated S) of every plane in g_xrot/g_srot
// ((nf, nx, ny, nz), the sweep's own frame), and the PCHIP ghost's partials in the
// bottom two unrotated planes in g_ghost (4, nf, nx, ny): chi(1), chi(2), S(1), S(2).
__global__ void __launch_bounds__(128) k_quad_rot_column_adj(int nf, int nx, int ny, int nz, const float *chi,
                                                             const float *S, const RotCol *rot, const int *slab_z0,
                                                             int nslab, QuadConst qc, PchipConst pc, float dtmax,
                                                             float Imax, const float *g_top, float *g_xrot,
                                                             float *g_srot, float *g_ghost) {
  const size_t plane = (size_t)nf * nx * ny;
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= plane) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  // ghost
  float d_c1, d_c2, d_s1, d_s2;
  const float gx0 = pchip_ghost_d(chi[g], chi[g + plane], pc, d_c1, d_c2);
  const float gs0 = pchip_ghost_d(S[g], S[g + plane], pc, d_s1, d_s2);
  // pass 1: forward, the intensity entering every slab (the slab-face checkpoints)
  float Ient[ADJ_MAXSLAB];
  {
    float gx = gx0, gs = gs0, gI = gs0;
    for (int s = 0; s < nslab; s++) {
      Ient[s] = gI;
      const int z0 = slab_z0[s], n = slab_z0[s + 1] - z0;
      float xu = gx, su = gs, Iu = gI, xc, sc, xd, sd;
      rot_at(chi, S, plane, z0, rot[z0], f, x, y, nf, nx, ny, xc, sc);
      rot_at(chi, S, plane, z0 + 1, rot[z0 + 1], f, x, y, nf, nx, ny, xd, sd);
      for (int zl = 1; zl < n; zl++) {
        Iu = quad_fwd<float>(xu, xc, xd, su, sc, sd, Iu, true, qc, dtmax, Imax);
        if (zl + 1 < n) {
          xu = xc; su = sc; xc = xd; sc = sd;
          rot_at(chi, S, plane, z0 + zl + 1, rot[z0 + zl + 1], f, x, y, nf, nx, ny, xd, sd);
        }
      }
      gI = quad_fwd<float>(xu, xc, xd, su, sc, sd, Iu, false, qc, dtmax, Imax);
      gx = xd; gs = sd;
    }
  }
  // pass 2: the slabs top to bottom, each recomputed from its face and reversed
  float xs[ADJ_MAXN], ss[ADJ_MAXN], Is[ADJ_MAXN], gxs[ADJ_MAXN], gss[ADJ_MAXN];
  float gI_exit = g_top[g], gx_exit = 0.0f, gs_exit = 0.0f;
  for (int s = nslab - 1; s >= 0; s--) {
    const int z0 = slab_z0[s], n = slab_z0[s + 1] - z0;
    float xe, se;
    if (s == 0) { xe = gx0; se = gs0; }
    else rot_at(chi, S, plane, z0 - 1, rot[z0 - 1], f, x, y, nf, nx, ny, xe, se);
    for (int k = 0; k < n; k++) {
      rot_at(chi, S, plane, z0 + k, rot[z0 + k], f, x, y, nf, nx, ny, xs[k], ss[k]);
      gxs[k] = 0.0f;
      gss[k] = 0.0f;
    }
    // forward intensities I_0 .. I_{n-2} of the interior steps
    for (int k = 0; k + 1 < n; k++) {
      const float xu = k == 0 ? xe : xs[k - 1], su = k == 0 ? se : ss[k - 1];
      const float Iu = k == 0 ? Ient[s] : Is[k - 1];
      Is[k] = quad_fwd<float>(xu, xs[k], xs[k + 1], su, ss[k], ss[k + 1], Iu, true, qc, dtmax, Imax);
    }
    gxs[n - 1] += gx_exit;
    gss[n - 1] += gs_exit;
    float gxe = 0.0f, gse = 0.0f;
    // the final step: the last interior step's three planes, I_{n-2} upstream
    float gIprev;
    {
      const int k = n - 2;
      const float xu = k == 0 ? xe : xs[k - 1], su = k == 0 ? se : ss[k - 1];
      QStepGrad<float> d = {0, 0, 0, 0, 0, 0, 0};
      quad_step_adj<float>(xu, xs[k], xs[k + 1], su, ss[k], ss[k + 1], Is[k], false, qc.rdsup, qc.dsup1, qc.dsup2,
                           dtmax, Imax, gI_exit, d);
      if (k == 0) { gxe += d.xu; gse += d.su; } else { gxs[k - 1] += d.xu; gss[k - 1] += d.su; }
      gxs[k] += d.xc; gss[k] += d.sc; gxs[k + 1] += d.xd; gss[k + 1] += d.sd;
      gIprev = d.Iu;
    }
    // the interior steps backwards
    for (int k = n - 2; k >= 0; k--) {
      const float xu = k == 0 ? xe : xs[k - 1], su = k == 0 ? se : ss[k - 1];
      const float Iu = k == 0 ? Ient[s] : Is[k - 1];
      QStepGrad<float> d = {0, 0, 0, 0, 0, 0, 0};
      quad_step_adj<float>(xu, xs[k], xs[k + 1], su, ss[k], ss[k + 1], Iu, true, qc.rdsup, qc.dsup1, qc.dsup2, dtmax,
                           Imax, gIprev, d);
      if (k == 0) { gxe += d.xu; gse += d.su; } else { gxs[k - 1] += d.xu; gss[k - 1] += d.su; }
      gxs[k] += d.xc; gss[k] += d.sc; gxs[k + 1] += d.xd; gss[k + 1] += d.sd;
      gIprev = d.Iu;
    }
    for (int k = 0; k < n; k++) {
      g_xrot[plane * (z0 + k) + g] = gxs[k];
      g_srot[plane * (z0 + k) + g] = gss[k];
    }
    // into the slab below: its exit plane's rotated values and exit intensity
    gI_exit = gIprev;
    gx_exit = gxe;
    gs_exit = gse;
  }
  // the ghost below the bottom slab: x = pchip(chi), s = I = pchip(S)
  const float gsum = gs_exit + gI_exit;
  g_ghost[g] = gx_exit * d_c1;
  g_ghost[g + plane] = gx_exit * d_c2;
  g_ghost[g + 2 * plane] = gsum * d_s1;
  g_ghost[g + 3 * plane] = gsum * d_s2;
}

// The transpose of the fused rotation: dL/dchi and dL/dS of every cell of the
// unrotated planes, gathered from the (up to) four columns whose bilinear taps read
// it, plus the ghost's terms in the bottom two planes.
__global__ void k_unrotate_adj(int nf, int nx, int ny, int nz, const RotCol *rot, const float *g_xrot,
                               const float *g_srot, const float *g_ghost, float *g_chi, float *g_S) {
  const size_t plane = (size_t)nf * nx * ny;
  const size_t n = plane * nz;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const size_t in = t % plane;
    const int z = (int)(t / plane);
    const int f = (int)(in % nf), x = (int)((in / nf) % nx), y = (int)(in / ((size_t)nf * nx));
    const RotCol r = rot[z];
    int xa = x - r.ux; xa = xa < 0 ? xa + nx : xa;          // columns whose first tap is x
    int xb = xa - 1; xb = xb < 0 ? xb + nx : xb;            // whose second tap is x
    int ya = y - r.uy; ya = ya < 0 ? ya + ny : ya;
    int yb = ya - 1; yb = yb < 0 ? yb + ny : yb;
    const size_t o = plane * z + f;
    auto at = [&](int cx, int cy) { return o + (size_t)nf * ((size_t)cx + (size_t)nx * cy); };
    float gc = r.a * g_xrot[at(xa, ya)] + r.b * g_xrot[at(xb, ya)] + r.c * g_xrot[at(xa, yb)] + r.d * g_xrot[at(xb, yb)];
    float gs = r.a * g_srot[at(xa, ya)] + r.b * g_srot[at(xb, ya)] + r.c * g_srot[at(xa, yb)] + r.d * g_srot[at(xb, yb)];
    if (z < 2) {
      gc += g_ghost[in + plane * z];
      gs += g_ghost[in + plane * (2 + z)];
    }
    g_chi[t] = gc;
    g_S[t] = gs;
  }
}

// The transfer units of every point from its line opacity chi_l (the opacity
// kernel's epilogue on its own): chil, chi, S (nf, ncell)
__global__ void k_units_fwd(int nf, int ncell, const double *nu, const float *temp, const float *chi_c,
                            float maser_chi_floor, const float *chil, float *chi, float *S) {
  const size_t n = (size_t)nf * ncell;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / nf), f = (int)(i % nf);
    const float T = temp[c];
    const float h_kT = (float)(M3D_H_K / (double)T);
    point_units(chi_c[c], h_kT, nu[f], chil[i], chil[i], maser_chi_floor, chi[i], S[i]);
  }
}

// The adjoint of the transfer units of one point: given dL/dchi, dL/dS and the line
// opacity chi_l, returns dL/dchi_l and adds the point's dL/dT and dL/dchi_c.
__device__ __forceinline__ float units_adj(float chi_c, float T, float h_kT, double nu, float chil, float fl, float g_chi,
                                           float g_S, float &g_T, float &g_chic) {
  const float hv = (float)(nu * (double)h_kT);
  float E, u0;
  exp_neg(hv, E, u0);
  const float beta = fmaxf(E, FLT_MIN);
  const float Bnu = beta / (1.0f - beta);
  const float eta_c = chi_c * Bnu;
  const float xhat = chi_c + eta_c;
  const float ehat = eta_c / beta;
  const float w1 = xhat + chil, w2 = ehat + chil;
  const float etav = w2 * beta;
  const float chi_raw = w1 - etav;
  const float floor_ = fmaxf(fl * fabsf(w1), FLT_MIN);
  const bool floored = fabsf(chi_raw) < floor_;
  const float chi = floored ? copysignf(floor_, chi_raw) : chi_raw;
  const float S = etav / chi;
  // S = etav / chi
  const float g_etav0 = g_S / chi;
  const float g_chi_t = g_chi - g_S * S / chi;
  float g_w1, g_etav;
  if (floored) {
    g_w1 = (fl * fabsf(w1) >= FLT_MIN) ? g_chi_t * fl * copysignf(1.0f, w1) * copysignf(1.0f, chi_raw) : 0.0f;
    g_etav = g_etav0;
  } else {
    g_w1 = g_chi_t;
    g_etav = g_etav0 - g_chi_t;
  }
  const float g_w2 = g_etav * beta;
  float g_beta = g_etav * w2;
  const float g_xhat = g_w1, g_ehat = g_w2;
  const float g_etac = g_xhat + g_ehat / beta;
  g_beta -= g_ehat * eta_c / (beta * beta);
  g_chic += g_xhat + g_etac * Bnu;
  const float g_Bnu = g_etac * chi_c;
  g_beta += g_Bnu / ((1.0f - beta) * (1.0f - beta));
  // beta = exp(-hv), hv = h nu/(k T): dbeta/dT = beta hv / T
  if (E > FLT_MIN) g_T += g_beta * beta * hv / T;
  return g_w1 + g_w2;
}

// k_units_adj: one thread per cell, its window's frequencies in order.  chil, g_chi,
// g_S: (nf, ncell); writes g_chil and adds into g_temp and g_chic.
__global__ void k_units_adj(int nf, int ncell, const double *nu, const float *temp, const float *chi_c,
                            float maser_chi_floor, const float *chil, const float *g_chi, const float *g_S,
                            float *g_chil, float *g_temp, float *g_chic) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const float T = temp[c], cc = chi_c[c];
    const float h_kT = (float)(M3D_H_K / (double)T);
    float gT = 0.0f, gC = 0.0f;
    for (int f = 0; f < nf; f++) {
      const size_t i = (size_t)f + (size_t)nf * c;
      g_chil[i] = units_adj(cc, T, h_kT, nu[f], chil[i], maser_chi_floor, g_chi[i], g_S[i], gT, gC);
    }
    g_temp[c] += gT;
    g_chic[c] += gC;
  }
}

// d ih / d D of qlg_setup's half-width factor ih = e/(gL e + SQ), e = D + 0.606 gL,
// SQ = sqrt(ln2) D^2
__device__ __forceinline__ float dih_dD(float gL, float D) {
  const float e = fmaf(gL, 0.60602209212341318f, D);
  const float den = fmaf(gL, e, 0.8325546112f * D * D);
  return (den - e * (gL + 2.0f * 0.8325546112f * D)) / (den * den);
}

// Per line: the partials of qlg_setup's coefficients in ih at fixed gL and S
struct QlgCoefD { float bL, gG, cZH, cL2; };
__device__ __forceinline__ QlgCoefD qlg_setup_dih(float gL, float S, const QlgCoef &c) {
  const float ih = c.ih, r = gL * ih, q = r * (1.0f - r), sc = S * ih, qs = q * sc, X = 2.0f * r - 1.0f;
  const float dr = gL, dsc = S, dq = gL * (1.0f - 2.0f * r), dqs = dq * sc + q * dsc, dX = 2.0f * gL;
  QlgCoefD d;
  d.bL = 0.3183098862f * (dr * sc + r * dsc);
  d.gG = dqs * fmaf(X, -0.11019326278794868f, -0.064924393191013452f) + qs * (-0.11019326278794868f) * dX +
         0.4697186f * (-dr * sc + (1.0f - r) * dsc);
  d.cZH = dqs * fmaf(X, -0.10567135279610407f, 0.38494195930078284f) + qs * (-0.10567135279610407f) * dX;
  d.cL2 = dqs * fmaf(X, 0.16241029253712097f, 0.04054415746208978f) + qs * 0.16241029253712097f * dX;
  return d;
}

// one profile point: K exactly as qlg_eval<MK> forms it, and dK/dih (the continuous
// member: G(u) = 2^-u, W' from the table's differences dW)
template <bool MK>
__device__ __forceinline__ float qlg_eval_d(const float2 *tab, const float *dW, const QlgCoef &c, const QlgCoefD &cd,
                                            float x, float &dK_dih) {
  const float xs = fabsf(x) * c.ih;
  const float u = xs * xs;
  const float L = qlg_rcp<MK>(1.0f + u);
  const float y = fminf(xs * 800.0f, 9019.0f);
  const int ig = qlg_node(y);
  const float2 gw = tab[ig];
  const float G = gw.x, W = gw.y;
  float p = fmaf(c.cZH, W, c.cL2);
  const float P = p;
  p = fmaf(L, p, c.bL);
  const float K = fmaf(L, p, G * c.gG);
  const float L2 = L * L;
  const float dK_du = fmaf(L2, fmaf(c.cZH, dW[ig], -fmaf(2.0f * L, P, c.bL)), -0.69314718f * G * c.gG);
  dK_dih = fmaf(dK_du, 2.0f * u / c.ih, fmaf(L, fmaf(L, fmaf(W, cd.cZH, cd.cL2), cd.bL), G * cd.gG));
  return K;
}

// One line's window replayed: chl gets the forward's K bit for bit (the forms the
// forward chooses by warp vote all give the general form's bits), Gl and Hl the sums
// of g_chil K and g_chil dK/dih.  FAR: every point beyond the table, whose last node
// gives G, W and W' at every point, so the per-point work is the forward's far form
// plus the derivative's few terms.
template <int NF, bool FULL, bool FAR, bool MK>
__device__ __forceinline__ void deposit_adj(float (&chl)[NF], const float (&gch)[NF], const float2 *s_tab,
                                            const float *s_dW, const QlgCoef &cf, const QlgCoefD &cd, float x0,
                                            float kfa, int fa, int fb, float &Gl, float &Hl) {
  if (FAR) {
    const float2 gw = s_tab[QLG_NTAB - 1];
    const float p1 = fmaf(cf.cZH, gw.y, cf.cL2);
    const float gg = gw.x * cf.gG;
    const float ca = cf.cZH * s_dW[QLG_NTAB - 1], cb = -0.69314718f * gg;
    const float e1 = fmaf(gw.y, cd.cZH, cd.cL2), e3 = gw.x * cd.gG;
    const float r2ih = 2.0f / cf.ih;
#pragma unroll
    for (int f = 0; f < NF; f++) {
      if (FULL || (f + 1 >= fa && f + 1 <= fb)) {
        const float xs = fabsf(x0 + (FULL ? (float)f : ((float)f + kfa))) * cf.ih;
        const float u = xs * xs;
        const float L = qlg_rcp<MK>(1.0f + u);
        const float K = fmaf(L, fmaf(L, p1, cf.bL), gg);
        chl[f] = fmaf(K, 1.0f, chl[f]);
        const float dK_du = fmaf(L * L, ca - fmaf(2.0f * L, p1, cf.bL), cb);
        const float dKi = fmaf(dK_du, u * r2ih, fmaf(L, fmaf(L, e1, cd.bL), e3));
        Gl = fmaf(gch[f], K, Gl);
        Hl = fmaf(gch[f], dKi, Hl);
      }
    }
  } else {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      if (FULL || (f + 1 >= fa && f + 1 <= fb)) {
        float dKi;
        const float K = qlg_eval_d<MK>(s_tab, s_dW, cf, cd, x0 + (FULL ? (float)f : ((float)f + kfa)), dKi);
        chl[f] = fmaf(K, 1.0f, chl[f]);
        Gl = fmaf(gch[f], K, Gl);
        Hl = fmaf(gch[f], dKi, Hl);
      }
    }
  }
}

template <int NF, bool MK>
__device__ __forceinline__ void deposit_adj_mk(float (&chl)[NF], const float (&gch)[NF], const float2 *s_tab,
                                               const float *s_dW, const QlgCoef &cf, const QlgCoefD &cd, float x0,
                                               float kfa, int fa, int fb, bool full, bool far, float &Gl, float &Hl) {
  if (far) {
    if (full) deposit_adj<NF, true, true, MK>(chl, gch, s_tab, s_dW, cf, cd, x0, kfa, fa, fb, Gl, Hl);
    else deposit_adj<NF, false, true, MK>(chl, gch, s_tab, s_dW, cf, cd, x0, kfa, fa, fb, Gl, Hl);
  } else {
    if (full) deposit_adj<NF, true, false, MK>(chl, gch, s_tab, s_dW, cf, cd, x0, kfa, fa, fb, Gl, Hl);
    else deposit_adj<NF, false, false, MK>(chl, gch, s_tab, s_dW, cf, cd, x0, kfa, fa, fb, Gl, Hl);
  }
}

// k_opacity_adj: the line loop of k_lte_opacity_units_lane<32> (no select_lines
// reach) replayed lane per cell with its decisions and its chi_l accumulation, each
// deposited point adding g_chil(f) K and g_chil(f) dK/dD.  Per depositing line: the
// sums go to dL/dlnbase (K is proportional to exp(arg)), dL/de_kT (-lower_ev times
// it), dL/dinv_df (through D = sdl/idf, in S = Rij D and the profile's width) and,
// reduced over the warp's cells and then the block, dL/dgpref of the line.
// Shared memory: the QLG tables (float2), the table differences dW, and the block's
// per-line sums (nline floats).
__global__ void __launch_bounds__(512, 1) k_opacity_adj(AtmosDev A, GridArgs G, const double *nu, double v0,
                                                        double v1, double v2, const float2 *tab, const float *dWg,
                                                        const float *g_chil, float *g_lnbase, float *g_ekt,
                                                        float *g_idf, float *const *g_gpref, int nline_max) {
  namespace cg = cooperative_groups;
  constexpr int NF = 32;
  extern __shared__ float smem[];
  float2 *s_tab = reinterpret_cast<float2 *>(smem);
  float *s_dW = smem + 2 * QLG_NTAB;
  float *s_gp = s_dW + QLG_NTAB;
  for (int i = threadIdx.x; i < QLG_NTAB; i += blockDim.x) {
    s_tab[i] = tab[i];
    s_dW[i] = dWg[i];
  }
  for (int i = threadIdx.x; i < A.nspecies * nline_max; i += blockDim.x) s_gp[i] = 0.0f;
  __syncthreads();
  const float ex_cutoff = -85.0f, voigt_peak = 0.5641895835f, sqrt_pi = 1.7724538509f;
  const float lt = logf_m3d(G.tol / voigt_peak);
  const int ncell = A.ncell;
  const int ncell_pad = (ncell + 31) / 32 * 32;
  const double llam_hi = G.llam[NF - 1];
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < ncell_pad; cell += gridDim.x * blockDim.x) {
    const bool live = cell < ncell;
    const int cs = live ? cell : ncell - 1;
    const float T = A.temp[cs], chi_c = A.chi_c[cs];
    const float h_kT = (float)(M3D_H_K / (double)T);
    float chl[NF], gch[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) {
      chl[f] = 0.0f;
      gch[f] = live ? g_chil[(size_t)f + (size_t)NF * cs] : 0.0f;
    }
    const float vproj = (float)((v0 * (double)A.vx[cs] + v1 * (double)A.vy[cs]) + v2 * (double)A.vz[cs]);
    const float ekt = A.e_kT[cs], ne = A.ne[cs], tothi = A.tothi[cs], starkpe = A.stark_pe[cs];
    const float x_lo = point_xhat(chi_c, h_kT, nu[0]), x_hi = point_xhat(chi_c, h_kT, nu[NF - 1]);
    const float lr_lo = x_lo > 0.0f ? lt + logf_m3d(x_lo) : -FLT_MAX;
    const float lr_hi = x_hi > 0.0f ? lt + logf_m3d(x_hi) : -FLT_MAX;
    float gE = 0.0f;
    for (int sp = 0; sp < A.nspecies; sp++) {
      const SpeciesDev &Sd = A.species[sp];
      const LineArgs &L = Sd.L;
      const float idf = Sd.inv_df[cs], base = Sd.lnbase[cs];
      const QlgCell qw = qlg_cell(G.sdl / idf);
      const float lvb2 = logf_m3d(Sd.vbar2[cs]);
      const float unsold_c = exp4(0.3f * lvb2) * tothi;
      float gB = 0.0f, gD = 0.0f;
      for (int l = 0; l < L.nline; l++) {
        if (L.active && !L.active[l]) continue;
        const float ex = L.lower_ev[l] * ekt;
        const float arg = (base + L.gpref[l]) - ex;
        if (arg < ex_cutoff) continue;
        const double llc = L.llam0[l] - (double)vproj;
        const double pos = (llc - G.llam1) * G.inv_dllam;
        const int ic = lround_d(pos) + 1;
        const int f0 = ic < 1 ? 1 : (ic > NF ? NF : ic);
        float cont0, lr0, chl0;
        if (f0 == 1) { cont0 = x_lo; lr0 = lr_lo; chl0 = chl[0]; }
        else if (f0 == NF) { cont0 = x_hi; lr0 = lr_hi; chl0 = chl[NF - 1]; }
        else {
          cont0 = point_xhat(chi_c, h_kT, nu[f0 - 1]);
          lr0 = cont0 > 0.0f ? lt + logf_m3d(cont0) : -FLT_MAX;
          chl0 = pick<NF>(chl, f0 - 1);
        }
        float refl = G.tol * cont0, lref;
        const float flo = G.flo_scale * chl0;
        if (flo > refl) { refl = flo; lref = logf_m3d(flo * sqrt_pi); }
        else lref = lr0;
        if (arg <= lref) continue;
        const float Rij = exp4(arg);
        if (voigt_peak * Rij <= refl) continue;
        const float a = line_damping_a(L, l, unsold_c, lvb2, tothi, ne, starkpe) * G.sdl;
        const float S = Rij * qw.D;
        const float x1 = f0 == 1 ? (float)(-pos)
                                 : (float)(((f0 == NF ? llam_hi : G.llam[f0 - 1]) - llc) * G.inv_dllam);
        const QlgCoef cf = qlg_setup(a, qw.D, qw.SQ, S);
        const float hw = qlg_halfwidth(qw, a, S, refl, arg - lref);
        const int noff = lround_pos(fminf(hw, (float)(NF + abs(ic))));
        const int fa = ic - noff > 1 ? ic - noff : 1;
        const int fb = ic + noff < NF ? ic + noff : NF;
        if (fa > fb) continue;
        const float x0 = x1 - (float)(f0 - fa);
        const float kfa = (float)(1 - fa);
        const QlgCoefD cd = qlg_setup_dih(a, S, cf);
        float Gl = 0.0f, Hl = 0.0f;
        // the forward's window forms, taken by the same warp votes
        const float xe = x0 + (float)(fb - fa);
        const float xnear = (x0 > 0.0f) ? x0 : ((xe < 0.0f) ? -xe : 0.0f);
        const unsigned conv = __activemask();
        const bool full = __all_sync(conv, fa == 1 && fb == NF);
        const bool far = __all_sync(conv, fminf((xnear * cf.ih) * 800.0f, 9019.0f) >= 9018.5f);
        const float xmax = fmaxf(fabsf(x0), fabsf(xe)) * cf.ih;
        if (__all_sync(conv, xmax <= 4611686018427387904.0f))
          deposit_adj_mk<NF, true>(chl, gch, s_tab, s_dW, cf, cd, x0, kfa, fa, fb, full, far, Gl, Hl);
        else
          deposit_adj_mk<NF, false>(chl, gch, s_tab, s_dW, cf, cd, x0, kfa, fa, fb, full, far, Gl, Hl);
        // K is proportional to S = Rij D: dK/dD = K/D + dK/dih dih/dD
        gB += Gl;
        gE -= L.lower_ev[l] * Gl;
        gD += Gl / qw.D + Hl * dih_dD(a, qw.D);
        cg::coalesced_group grp = cg::coalesced_threads();
        const float tot = cg::reduce(grp, Gl, cg::plus<float>());
        if (grp.thread_rank() == 0) atomicAdd(&s_gp[sp * nline_max + l], tot);
      }
      if (live) {
        g_lnbase[(size_t)sp * ncell + cs] += gB;
        // D = sdl / idf
        g_idf[(size_t)sp * ncell + cs] += gD * (-qw.D / idf);
      }
    }
    if (live) g_ekt[cs] += gE;
  }
  __syncthreads();
  for (int sp = 0; sp < A.nspecies; sp++)
    for (int i = threadIdx.x; i < A.species[sp].L.nline; i += blockDim.x) {
      const float v = s_gp[sp * nline_max + i];
      if (v != 0.0f) atomicAdd(g_gpref[sp] + i, v);
    }
}

}  // namespace m3d

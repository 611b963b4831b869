// The LTE synthesis output pass (rt_patch_t%execute do_final branch,
// rt_patch_mod.f90:1014-1030) as two kernels per ray direction:
//
//   k_lte_opacity_units  warp per cell: LTE background (beta, Bnu), work units
//                        (xhat, ehat), logref, the line opacity of every species in
//                        line order, and work_to_transfer_units -> (chi, Snu)
//   k_quad_rot_column    thread per (f, x, y): the whole column bottom to top, slab
//                        by slab, with rotate_array fused into the loads, the
//                        PCHIP ghost below the bottom slab, long_char_quadratic,
//                        and the exit plane of each slab handed to the next in
//                        registers; only the emergent plane is written.
#pragma once
#include "m3d_kernels.cuh"

namespace m3d {

struct SpeciesDev {
  LineArgs L;
  const float *inv_df, *vbar2, *lnbase;
};

struct AtmosDev {
  int ncell;
  const float *temp, *chi_c, *vx, *vy, *vz, *e_kT, *ne, *tothi, *stark_pe;
  int nspecies;
  const SpeciesDev *species;
  float maser_chi_floor;
};

// Work units and transfer units of one point, FP32 (rt_patch_mod.f90:2004-2023,
// 2309-2326, 3518-3536, 3571-3651, composition_mod.f90:1848-1858)
__device__ __forceinline__ void point_units(float chi_c, float h_kT, double nu, float chil, float etal, float fl,
                                            float &chi_out, float &S_out) {
  const float hv = (float)(nu * (double)h_kT);
  float E, u0;
  exp_neg(hv, E, u0);
  const float beta = fmaxf(E, FLT_MIN);
  const float Bnu = beta / (1.0f - beta);
  const float eta_c = chi_c * Bnu;
  const float xhat = chi_c + eta_c;
  const float ehat = eta_c / beta;
  const float w1 = xhat + chil;
  const float w2 = ehat + etal;
  const float etav = w2 * beta;
  float chi = w1 - etav;
  const float floor_ = fmaxf(fl * fabsf(w1), FLT_MIN);
  if (fabsf(chi) < floor_) chi = copysignf(floor_, chi);
  chi_out = chi;
  S_out = etav / chi;
}

// The same in FP64 (the plain FP64 path): beta and 1-beta from exp/expm1
__device__ __forceinline__ void point_units(double chi_c, double T, double nu, double chil, double etal, double fl,
                                            double &chi_out, double &S_out) {
  const double hv = nu * (M3D_H_K / T);
  const double beta = fmax(exp(-hv), DBL_MIN);
  const double omb = -expm1(-hv);
  const double Bnu = beta / omb;
  const double eta_c = chi_c * Bnu;
  const double xhat = chi_c + eta_c;
  const double ehat = eta_c / beta;
  const double w1 = xhat + chil;
  const double w2 = ehat + etal;
  const double etav = w2 * beta;
  double chi = w1 - etav;
  const double floor_ = fmax(fl * fabs(w1), DBL_MIN);
  if (fabs(chi) < floor_) chi = copysign(floor_, chi);
  chi_out = chi;
  S_out = etav / chi;
}

// xhat at one frequency, the tolerance reference of the line kernel
__device__ __forceinline__ float point_xhat(float chi_c, float h_kT, double nu) {
  const float hv = (float)(nu * (double)h_kT);
  float E, u0;
  exp_neg(hv, E, u0);
  const float beta = fmaxf(E, FLT_MIN);
  const float Bnu = beta / (1.0f - beta);
  return chi_c + chi_c * Bnu;
}

// Shared memory: the two QLG tables, then per warp xhat, logref, chi_l, eta_l (nf each)
template <typename TO>
__global__ void __launch_bounds__(256) k_lte_opacity_units(AtmosDev A, GridArgs G, const double *nu, double v0,
                                                           double v1, double v2, TO *chi_out, TO *S_out,
                                                           const float2 *tab) {
  extern __shared__ float smem[];
  float2 *s_tab = reinterpret_cast<float2 *>(smem);
  stage_tables(s_tab, tab);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const int nf = G.nf;
  const float lt = logf_m3d(G.tol / 0.5641895835f);
  float *s_x = smem + 2 * QLG_NTAB + (size_t)wid * 4 * nf;
  float *s_lr = s_x + nf, *s_chi = s_lr + nf, *s_eta = s_chi + nf;
  for (int cell = blockIdx.x * warps + wid; cell < A.ncell; cell += gridDim.x * warps) {
    const float T = A.temp[cell], chi_c = A.chi_c[cell];
    const float h_kT = (float)(M3D_H_K / (double)T);
    for (int f = lane; f < nf; f += 32) {
      const float xh = point_xhat(chi_c, h_kT, nu[f]);
      s_x[f] = xh;
      s_lr[f] = xh > 0.0f ? lt + logf_m3d(xh) : -FLT_MAX;
      s_chi[f] = 0.0f;
      s_eta[f] = 0.0f;
    }
    __syncwarp();
    CellArgs c;
    c.vproj = (float)((v0 * (double)A.vx[cell] + v1 * (double)A.vy[cell]) + v2 * (double)A.vz[cell]);
    c.ekt = A.e_kT[cell]; c.ne = A.ne[cell]; c.tothi = A.tothi[cell]; c.starkpe = A.stark_pe[cell];
    for (int sp = 0; sp < A.nspecies; sp++) {
      const SpeciesDev &S = A.species[sp];
      c.idf = S.inv_df[cell]; c.vbar2 = S.vbar2[cell]; c.base = S.lnbase[cell];
      auto dep = [](int) { return 1.0f; };
      warp_cell_lines(S.L, G, c, s_chi, s_eta, s_x, s_lr, dep, false, false, nullptr, nullptr, nullptr, s_tab,
                      lane);
    }
    __syncwarp();
    for (int f = lane; f < nf; f += 32) {
      TO co, so;
      if constexpr (sizeof(TO) == 4) {
        point_units(chi_c, h_kT, nu[f], s_chi[f], s_eta[f], A.maser_chi_floor, co, so);
      } else {
        point_units((double)chi_c, (double)T, nu[f], (double)s_chi[f], (double)s_eta[f], (double)A.maser_chi_floor, co, so);
      }
      chi_out[(size_t)f + (size_t)nf * cell] = co;
      S_out[(size_t)f + (size_t)nf * cell] = so;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// The same pass with one LANE per cell, for windows of NF frequencies: each lane
// runs its own cell's line loop in line order and keeps chi_l of the window in
// registers, so no lane idles on the per-line scalar work and every line's window
// is evaluated with one point per unrolled step.  In this LTE pass every line
// deposits the same profile into chi_l and eta_l (b_i = b_j = 1, both start at
// zero), so eta_l is chi_l and is not carried separately.  The tolerance
// reference at a line's nearest node f0 -- xhat and its log -- is kept for the two
// window edges, where every line centred outside the window lands, and formed on
// the spot otherwise; the accumulated line opacity there is picked out of the
// register array.  Results are bit-identical to k_lte_opacity_units.
// ---------------------------------------------------------------------------
// One line's profile over the window into chl.  far: every window point lies
// beyond the QLG table, where G and W are the last node's at every point and the
// evaluation is qlg_eval's with them folded in; full: the line covers the whole
// window, which then runs without per-point predicates (with fa = 1 the offset
// (float)f + kfa is (float)f).  MK: every point's 1 + xs^2 is below 2^126, so the
// reciprocal is rcp_markstein's.  All forms give the bits of the general one.
template <int NF, bool MK>
__device__ __forceinline__ void deposit_window(float (&chl)[NF], const float2 *s_tab, const QlgCoef &cf, float x0,
                                               float kfa, int fa, int fb, bool full, bool far) {
  if (far) {
    const float2 gw = s_tab[QLG_NTAB - 1];
    const float p1 = fmaf(cf.cZH, gw.y, cf.cL2);
    const float gg = gw.x * cf.gG;
    if (full) {
#pragma unroll
      for (int f = 0; f < NF; f++) {
        const float xs = fabsf(x0 + (float)f) * cf.ih;
        const float L = qlg_rcp<MK>(1.0f + xs * xs);
        const float K = fmaf(L, fmaf(L, p1, cf.bL), gg);
        chl[f] = fmaf(K, 1.0f, chl[f]);
      }
    } else {
#pragma unroll
      for (int f = 0; f < NF; f++) {
        if (f + 1 >= fa && f + 1 <= fb) {
          const float xs = fabsf(x0 + ((float)f + kfa)) * cf.ih;
          const float L = qlg_rcp<MK>(1.0f + xs * xs);
          const float K = fmaf(L, fmaf(L, p1, cf.bL), gg);
          chl[f] = fmaf(K, 1.0f, chl[f]);
        }
      }
    }
  } else if (full) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      const float K = qlg_eval<MK>(s_tab, cf, x0 + (float)f);
      chl[f] = fmaf(K, 1.0f, chl[f]);
    }
  } else {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      if (f + 1 >= fa && f + 1 <= fb) {
        const float K = qlg_eval<MK>(s_tab, cf, x0 + ((float)f + kfa));
        chl[f] = fmaf(K, 1.0f, chl[f]);
      }
    }
  }
}

// The same deposit, two window points per instruction (packed f32x2 arithmetic,
// each half rounded as the scalar form rounds it), for windows whose every 1 + xs^2
// is below 2^126 (the Markstein reciprocal).  Exact rewrites beside the packing:
//  * xs is formed with its sign, x ih; only xs^2 and |xs| are used, and the rounded
//    product is symmetric in the sign;
//  * d = 1 + xs^2 is formed per half in scalar (a packed product feeding a packed
//    sum was fused into one rounding by the code generator, which left K 1-2 ulp off
//    at a few points of about one table-form window in 10^4), and -d enters the
//    Newton step;
//  * the snapped node nint(min(|xs| 800, 9019)) is floor(RZ(y + 0.5)): rounding
//    toward zero never carries a positive sum past the integer below it, so this is
//    round-half-up of y >= 0, i.e. nint, with no special case below y = 0.5.  Adding
//    2^23 toward zero then leaves that integer in the low mantissa bits, so the
//    node's shared-memory address is one shift-add from the sum's bits.
// Points outside a partial window add +0; the running sum is never -0 (it starts at
// +0, and in round-to-nearest a sum is -0 only when both terms are), so adding +0
// leaves it unchanged, exactly as skipping the point does.
__device__ __forceinline__ float rcp_approx(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  return r;
}

__device__ __forceinline__ float2 lds_node(unsigned addr) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}

template <int NF, bool FULL, bool FAR>
__device__ __forceinline__ void deposit_window_x2(float (&chl)[NF], const float2 *s_tab, const QlgCoef &cf,
                                                  float x0, float kfa, int fa, int fb) {
  static_assert(NF % 2 == 0, "pairs of window points");
  const f32x2 X0 = splat2(x0), IH = splat2(cf.ih), ONE = splat2(1.0f), BL = splat2(cf.bL);
  const f32x2 KF = splat2(kfa);
  f32x2 P1 = 0, GG = 0, CZH = 0, CL2 = 0, GGc = 0;
  unsigned base = 0;
  if (FAR) {
    const float2 gw = s_tab[QLG_NTAB - 1];
    P1 = splat2(fmaf(cf.cZH, gw.y, cf.cL2));
    GG = splat2(gw.x * cf.gG);
  } else {
    CZH = splat2(cf.cZH);
    CL2 = splat2(cf.cL2);
    GGc = splat2(cf.gG);
    // node i sits at byte 8 i; the sum's bits are 0x4B000000 + i
    base = (unsigned)__cvta_generic_to_shared(s_tab) - (0x4B000000u << 3);
  }
#pragma unroll
  for (int k = 0; k < NF / 2; k++) {
    f32x2 F = pk2((float)(2 * k), (float)(2 * k + 1));
    if (!FULL) F = add2(F, KF);  // (float)f + kfa, exact
    const f32x2 x = add2(X0, F);
    const f32x2 xs = mul2(x, IH);
    float xa, xb;
    up2(xs, xa, xb);
    // 1 + xs^2 in scalar: the code generator fuses a packed product into the packed
    // sum that consumes it (one rounding where the reference rounds twice), which
    // the scalar forms under -fmad=false never are
    const float da = 1.0f + xa * xa, db = 1.0f + xb * xb;
    const f32x2 nd = pk2(-da, -db);
    const f32x2 r = pk2(rcp_approx(da), rcp_approx(db));
    const f32x2 e = fma2(nd, r, ONE);
    const f32x2 L = fma2(r, e, r);
    f32x2 K;
    if (FAR) {
      K = fma2(L, fma2(L, P1, BL), GG);
    } else {
      const f32x2 y = pk2(fminf(fabsf(xa) * 800.0f, 9019.0f), fminf(fabsf(xb) * 800.0f, 9019.0f));
      const f32x2 v = add2_rz(add2_rz(y, splat2(0.5f)), splat2(8388608.0f));
      float va, vb;
      up2(v, va, vb);
      const float2 ga = lds_node(base + (__float_as_uint(va) << 3));
      const float2 gb = lds_node(base + (__float_as_uint(vb) << 3));
      f32x2 p = fma2(CZH, pk2(ga.y, gb.y), CL2);
      p = fma2(L, p, BL);
      K = fma2(L, p, mul2(pk2(ga.x, gb.x), GGc));
    }
    if (!FULL) {
      float ka, kb;
      up2(K, ka, kb);
      ka = (2 * k + 1 >= fa && 2 * k + 1 <= fb) ? ka : 0.0f;
      kb = (2 * k + 2 >= fa && 2 * k + 2 <= fb) ? kb : 0.0f;
      K = pk2(ka, kb);
    }
    float lo, hi;
    up2(add2(K, pk2(chl[2 * k], chl[2 * k + 1])), lo, hi);
    chl[2 * k] = lo;
    chl[2 * k + 1] = hi;
  }
}

template <int NF>
__device__ __forceinline__ void deposit_window_mk(float (&chl)[NF], const float2 *s_tab, const QlgCoef &cf, float x0,
                                                  float kfa, int fa, int fb, bool full, bool far) {
  if (far) {
    if (full) deposit_window_x2<NF, true, true>(chl, s_tab, cf, x0, kfa, fa, fb);
    else deposit_window_x2<NF, false, true>(chl, s_tab, cf, x0, kfa, fa, fb);
  } else {
    if (full) deposit_window_x2<NF, true, false>(chl, s_tab, cf, x0, kfa, fa, fb);
    else deposit_window_x2<NF, false, false>(chl, s_tab, cf, x0, kfa, fa, fb);
  }
}

// lround of a double (half away from zero) for |x| < 2^31: floor(|x| + 0.5) with the
// sum rounded toward zero, which never reaches the next integer below the exact sum
// (an integer below 2^53 is representable), so it is exact; the conversion truncates.
__device__ __forceinline__ int lround_d(double x) {
  const int m = __double2int_rz(__dadd_rz(fabs(x), 0.5));
  return x < 0.0 ? -m : m;
}

// lroundf of v >= 0, the same way in float (above 2^23 v is an integer and stays)
__device__ __forceinline__ int lround_pos(float v) { return __float2int_rz(__fadd_rz(v, 0.5f)); }

template <int NF>
__device__ __forceinline__ float pick(const float (&a)[NF], int i) {
  float v = a[0];
#pragma unroll
  for (int k = 1; k < NF; k++) v = (k == i) ? a[k] : v;
  return v;
}

// REACH: the line list carries reach_in (has_reach): the lines select_lines kept,
// and lines centred beyond the window take the unfloored reference at the nearer
// end, no peak test and a window capped by their reach (linelist_mod.f90:844-854, 914-921)
// CHIL: write the line opacity chi_l of the window itself to chi_out (S_out unused):
// the input of the adjoint's transfer units
// BATCH: nray directions (vr, 3 each) and nwin windows of NF frequencies in one
// launch, each window with its own grid Gw[w] and frequencies nu + w NF; the warps run
// over (ray, window, cell) with the cells of a window padded to whole warps, so a warp
// holds one ray and window, and a cell's row of every window goes to chi_out +
// ray ncell nwin NF + nwin NF cell + w NF: per ray the rows of one window of nwin NF
// frequencies, which the column solvers take as they are
template <int NF, typename TO, bool REACH, bool CHIL = false, bool BATCH = false>
__global__ void __launch_bounds__(768, 1) k_lte_opacity_units_lane(AtmosDev A, GridArgs G0, const double *nu0,
                                                                   double v0_, double v1_, double v2_, TO *chi_out,
                                                                   TO *S_out, const float2 *tab, const GridArgs *Gw,
                                                                   int nwin, const double *vr, int nray) {
  extern __shared__ float smem[];
  float2 *s_tab = reinterpret_cast<float2 *>(smem);
  stage_tables(s_tab, tab);
  const float ex_cutoff = -85.0f, voigt_peak = 0.5641895835f, sqrt_pi = 1.7724538509f;
  const float lt = logf_m3d(G0.tol / voigt_peak);
  const int ncell = A.ncell;
  const int nthreads = gridDim.x * blockDim.x;
  const int ncell_pad = (ncell + 31) / 32 * 32;
  const int nvc = BATCH ? ncell_pad * nwin * nray : ncell_pad;
  for (int vc = blockIdx.x * blockDim.x + threadIdx.x; vc < nvc; vc += nthreads) {
    const int ray = BATCH ? vc / (ncell_pad * nwin) : 0;
    const int wc = BATCH ? vc - ray * (ncell_pad * nwin) : vc;
    const int w = BATCH ? wc / ncell_pad : 0;
    const int cell = BATCH ? wc - w * ncell_pad : wc;
    const GridArgs G = BATCH ? Gw[w] : G0;
    const double *nu = BATCH ? nu0 + (size_t)NF * w : nu0;
    const double v0 = BATCH ? vr[3 * ray] : v0_, v1 = BATCH ? vr[3 * ray + 1] : v1_, v2 = BATCH ? vr[3 * ray + 2] : v2_;
    const size_t row = BATCH ? (size_t)ray * ncell * nwin * NF + (size_t)NF * nwin * cell + (size_t)NF * w
                             : (size_t)NF * cell;
    const bool live = cell < ncell;
    const int cs = live ? cell : ncell - 1;
    const float T = A.temp[cs], chi_c = A.chi_c[cs];
    const float h_kT = (float)(M3D_H_K / (double)T);
    float chl[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) chl[f] = 0.0f;
    const float vproj = (float)((v0 * (double)A.vx[cs] + v1 * (double)A.vy[cs]) + v2 * (double)A.vz[cs]);
    const float ekt = A.e_kT[cs], ne = A.ne[cs], tothi = A.tothi[cs], starkpe = A.stark_pe[cs];
    // xhat and logref at the window edges
    const float x_lo = point_xhat(chi_c, h_kT, nu[0]), x_hi = point_xhat(chi_c, h_kT, nu[NF - 1]);
    const float lr_lo = x_lo > 0.0f ? lt + logf_m3d(x_lo) : -FLT_MAX;
    const float lr_hi = x_hi > 0.0f ? lt + logf_m3d(x_hi) : -FLT_MAX;
    const double llam_hi = G.llam[NF - 1];
    for (int sp = 0; sp < A.nspecies; sp++) {
      const SpeciesDev &Sd = A.species[sp];
      const LineArgs &L = Sd.L;
      const float idf = Sd.inv_df[cs], base = Sd.lnbase[cs];
      const QlgCell qw = qlg_cell(G.sdl / idf);
      const float lvb2 = logf_m3d(Sd.vbar2[cs]);
      const float unsold_c = exp4(0.3f * lvb2) * tothi;
      const int nline = REACH ? *L.nsel : L.nline;
      for (int s = 0; s < nline; s++) {
        const int l = REACH ? L.sel[s] : s;
        if (L.active && !L.active[l]) continue;
        const float ex = L.lower_ev[l] * ekt;
        const float arg = (base + L.gpref[l]) - ex;
        if (arg < ex_cutoff) continue;
        const double llc = L.llam0[l] - (double)vproj;
        const double pos = (llc - G.llam1) * G.inv_dllam;
        const int ic = lround_d(pos) + 1;
        const int f0 = ic < 1 ? 1 : (ic > NF ? NF : ic);
        // the nearest node's xhat, its log and the line opacity there: a line centred
        // outside the window -- nearly all of them -- lands on an edge, whose values
        // are at hand; an interior node forms them (one branch, taken rarely)
        float cont0, lr0, chl0;
        if (f0 == 1) { cont0 = x_lo; lr0 = lr_lo; chl0 = chl[0]; }
        else if (f0 == NF) { cont0 = x_hi; lr0 = lr_hi; chl0 = chl[NF - 1]; }
        else {
          cont0 = point_xhat(chi_c, h_kT, nu[f0 - 1]);
          lr0 = cont0 > 0.0f ? lt + logf_m3d(cont0) : -FLT_MAX;
          chl0 = pick<NF>(chl, f0 - 1);
        }
        float refl = G.tol * cont0;
        float lref, cap = FLT_MAX;
        const bool outside = REACH && (llc < G.llam[0] || llc > llam_hi);
        if (outside) {
          lref = lr0;
          if (arg <= lref) continue;
          cap = (float)((double)L.reach_in[l] * G.inv_dllam);
        } else {
          const float flo = G.flo_scale * chl0;
          if (flo > refl) { refl = flo; lref = logf_m3d(flo * sqrt_pi); }
          else lref = lr0;
          if (arg <= lref) continue;
        }
        const float Rij = exp4(arg);
        if (!outside && voigt_peak * Rij <= refl) continue;
        const float a = line_damping_a(L, l, unsold_c, lvb2, tothi, ne, starkpe) * G.sdl;
        const float S = Rij * qw.D;
        // (llam(f0) - llc)/dllam; at f0 = 1 it is -pos exactly (the rounded difference
        // and product are odd in their sign)
        const float x1 = f0 == 1 ? (float)(-pos)
                                 : (float)(((f0 == NF ? llam_hi : G.llam[f0 - 1]) - llc) * G.inv_dllam);
        const QlgCoef cf = qlg_setup(a, qw.D, qw.SQ, S);
        const float hw = qlg_halfwidth(qw, a, S, refl, arg - lref);
        const int noff = lround_pos(fminf(fminf(hw, cap), (float)(NF + abs(ic))));
        const int fa = ic - noff > 1 ? ic - noff : 1;
        const int fb = ic + noff < NF ? ic + noff : NF;
        if (fa > fb) continue;
        const float x0 = x1 - (float)(f0 - fa);
        const float kfa = (float)(1 - fa);    // (float)(f + 1 - fa) = (float)f + kfa, exactly
        // Far wing: when even the window point nearest the line centre snaps to the
        // last table node, G and W are the same two constants at every point, and the
        // evaluation is qlg_eval's with them folded in.  The snapped index is monotone
        // in |x| (rounded products are monotone), so the nearer window end decides.
        const float xe = x0 + (float)(fb - fa);
        const float xnear = (x0 > 0.0f) ? x0 : ((xe < 0.0f) ? -xe : 0.0f);
        // A window over the whole frequency range -- most lines -- runs without
        // per-point predicates, and with fa = 1 the offset (float)f + kfa is (float)f.
        // The far-wing and whole-window forms are taken only when every converged
        // lane of the warp qualifies: the general forms give the same values where
        // the special ones apply, so the warp never runs two forms of one line.
        const unsigned conv = __activemask();
        const bool full = __all_sync(conv, fa == 1 && fb == NF);
        const bool far = __all_sync(conv, fminf((xnear * cf.ih) * 800.0f, 9019.0f) >= 9018.5f);
        // The window's largest |x| ih bounds every point's 1 + xs^2 (rounded products
        // are monotone): at most 2^62 keeps it under 2^126, where rcp_markstein is
        // exact.  One vote per line picks the reciprocal for the whole window.
        const float xmax = fmaxf(fabsf(x0), fabsf(xe)) * cf.ih;
        if (__all_sync(conv, xmax <= 4611686018427387904.0f))
          deposit_window_mk<NF>(chl, s_tab, cf, x0, kfa, fa, fb, full, far);
        else
          deposit_window<NF, false>(chl, s_tab, cf, x0, kfa, fa, fb, full, far);
      }
    }
    if (CHIL) {
      if (live) {
        float *co = reinterpret_cast<float *>(chi_out) + row;
#pragma unroll
        for (int f = 0; f < NF; f += 4)
          *reinterpret_cast<float4 *>(co + f) = make_float4(chl[f], chl[f + 1], chl[f + 2], chl[f + 3]);
      }
      continue;
    }
    // epilogue: transfer units, written as 16-byte stores of this cell's row
    if (live) {
      TO *co = chi_out + row, *so = S_out + row;
#pragma unroll
      for (int f = 0; f < NF; f += 4) {
        TO c4[4], s4[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if constexpr (sizeof(TO) == 4) {
            point_units(chi_c, h_kT, nu[f + k], chl[f + k], chl[f + k], A.maser_chi_floor, c4[k], s4[k]);
          } else {
            point_units((double)chi_c, (double)T, nu[f + k], (double)chl[f + k], (double)chl[f + k],
                        (double)A.maser_chi_floor, c4[k], s4[k]);
          }
        }
        if constexpr (sizeof(TO) == 4) {
          *reinterpret_cast<float4 *>(co + f) = make_float4(c4[0], c4[1], c4[2], c4[3]);
          *reinterpret_cast<float4 *>(so + f) = make_float4(s4[0], s4[1], s4[2], s4[3]);
        } else {
          reinterpret_cast<double2 *>(co + f)[0] = make_double2(c4[0], c4[1]);
          reinterpret_cast<double2 *>(co + f)[1] = make_double2(c4[2], c4[3]);
          reinterpret_cast<double2 *>(so + f)[0] = make_double2(s4[0], s4[1]);
          reinterpret_cast<double2 *>(so + f)[1] = make_double2(s4[2], s4[3]);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The plain FP64 path of the same pass: the line opacity, the QLG-bot profile and
// the transfer units all in double.  One lane per cell, chi_l of the window in
// double registers, the general window form (per-point predicates) for every line.
// The algorithm is the FP32 pass's step for step; what changes is the arithmetic:
//  * the tables TGX = 2^-u and TH2X = Z_0.2(u)(1+u)^2 are the fp64 values of
//    qlg_init's formulas (not rounded to float), read from global memory;
//  * the QLG-bot constants are the exact values the fitted float parameters stand
//    for (1/pi, sqrt(ln2/pi), sqrt(ln2), 1/sqrt(pi)); the fit's own coefficients are
//    the published digits;
//  * exp and log are the device's double exp/log (Rij, the damping power, logref);
//  * vproj, the tolerance references and xhat are formed in double.
// It is the accuracy reference the FP32 pass is measured against.
// ---------------------------------------------------------------------------
struct QlgCoef64 { double ih, bL, gG, cZH, cL2; };

__device__ __forceinline__ QlgCoef64 qlg_setup64(double gL, double D, double SQ, double S) {
  QlgCoef64 c;
  const double e = fma(gL, 0.60602209212341318, D);
  c.ih = e / fma(gL, e, SQ);
  const double r = gL * c.ih;
  const double q = r * (1.0 - r);
  const double sc = S * c.ih;
  const double qs = q * sc;
  const double x = 2.0 * r - 1.0;
  c.bL = (0.31830988618379067 * r) * sc;
  c.gG = fma(qs, fma(x, -0.11019326278794868, -0.064924393191013452), (0.46971863934982566 * (1.0 - r)) * sc);
  c.cZH = qs * fma(x, -0.10567135279610407, 0.38494195930078284);
  c.cL2 = qs * fma(x, 0.16241029253712097, 0.04054415746208978);
  return c;
}

__device__ __forceinline__ double qlg_eval64(const double2 *tab, const QlgCoef64 &c, double x) {
  const double xs = fabs(x) * c.ih;
  const double u = xs * xs;
  const double L = 1.0 / (1.0 + u);
  const int ig = (int)lround(fmin(xs * 800.0, 9019.0));
  const double2 gw = __ldg(tab + ig);
  double p = fma(c.cZH, gw.y, c.cL2);
  p = fma(L, p, c.bL);
  return fma(L, p, gw.x * c.gG);
}

__device__ __forceinline__ double qlg_halfwidth64(double D2, double gL, double S, double ref, double lnq) {
  const double AL = ((0.31830988618379067 * gL) * S) / ref;
  const double h1 = fma(D2, lnq, fmin(AL, 1.5 * D2));
  const double h2 = (AL - fmax(fma(gL, gL, -0.5 * D2), 0.0)) + fmin(AL, 5.0 * D2);
  return sqrt(fmax(fmax(h1, h2), 0.0));
}

__device__ __forceinline__ double point_xhat64(double chi_c, double T, double nu) {
  const double hv = nu * (M3D_H_K / T);
  const double beta = fmax(exp(-hv), DBL_MIN);
  const double Bnu = beta / (-expm1(-hv));
  return chi_c + chi_c * Bnu;
}

// chi_l of a window: NF > 0 in registers; NF = 0 (any window size) in the cell's
// row of chi_out, which the epilogue then overwrites with the transfer units
template <int NF>
struct ChlF64 {
  double v[NF];
  __device__ __forceinline__ ChlF64(double *) {}
  __device__ __forceinline__ double &operator[](int i) { return v[i]; }
};
template <>
struct ChlF64<0> {
  double *p;
  __device__ __forceinline__ ChlF64(double *row) : p(row) {}
  __device__ __forceinline__ double &operator[](int i) { return p[i]; }
};

// BATCH: nray directions and nwin windows in one launch, as
// k_lte_opacity_units_lane<..., BATCH> (NF > 0)
template <int NF, bool BATCH = false>
__global__ void __launch_bounds__(256) k_lte_opacity_units_f64(AtmosDev A, GridArgs G0, const double *nu0,
                                                               double v0_, double v1_, double v2_, double *chi_out,
                                                               double *S_out, const double2 *tab, const GridArgs *Gw,
                                                               int nwin, const double *vr, int nray) {
  static_assert(!BATCH || NF > 0, "window batches of a fixed window size");
  const double ex_cutoff = -85.0, voigt_peak = 0.56418958354775628, sqrt_pi = 1.7724538509055160;
  const double tol = (double)G0.tol, flo_scale = (double)G0.flo_scale;
  const double lt = log(tol / voigt_peak);
  const int ncell = A.ncell;
  const int nf = NF > 0 ? NF : G0.nf;
  const int nvc = BATCH ? ncell * nwin * nray : ncell;
  for (int vc = blockIdx.x * blockDim.x + threadIdx.x; vc < nvc; vc += gridDim.x * blockDim.x) {
    const int ray = BATCH ? vc / (ncell * nwin) : 0;
    const int wc = BATCH ? vc - ray * (ncell * nwin) : vc;
    const int w = BATCH ? wc / ncell : 0;
    const int cell = BATCH ? wc - w * ncell : wc;
    const GridArgs G = BATCH ? Gw[w] : G0;
    const double *nu = BATCH ? nu0 + (size_t)nf * w : nu0;
    const double v0 = BATCH ? vr[3 * ray] : v0_, v1 = BATCH ? vr[3 * ray + 1] : v1_, v2 = BATCH ? vr[3 * ray + 2] : v2_;
    const double sdl = G.inv_dllam;
    const double T = A.temp[cell], chi_c = A.chi_c[cell];
    const size_t row = BATCH ? (size_t)ray * ncell * nwin * nf + (size_t)nf * nwin * cell + (size_t)nf * w
                             : (size_t)nf * cell;
    double *co = chi_out + row, *so = S_out + row;
    ChlF64<NF> chl(co);
#pragma unroll
    for (int f = 0; f < nf; f++) chl[f] = 0.0;
    const double vproj = (v0 * (double)A.vx[cell] + v1 * (double)A.vy[cell]) + v2 * (double)A.vz[cell];
    const double ekt = A.e_kT[cell], ne = A.ne[cell], tothi = A.tothi[cell], starkpe = A.stark_pe[cell];
    // xhat and logref at the window edges, where every line centred outside lands
    const double x_lo = point_xhat64(chi_c, T, nu[0]), x_hi = point_xhat64(chi_c, T, nu[nf - 1]);
    const double lr_lo = x_lo > 0.0 ? lt + log(x_lo) : -DBL_MAX, lr_hi = x_hi > 0.0 ? lt + log(x_hi) : -DBL_MAX;
    for (int sp = 0; sp < A.nspecies; sp++) {
      const SpeciesDev &Sd = A.species[sp];
      const LineArgs &L = Sd.L;
      const double idf = Sd.inv_df[cell], base = Sd.lnbase[cell];
      const double D = sdl / idf, D2 = D * D, SQ = 0.83255461115769776 * D2;
      const double lvb2 = log((double)Sd.vbar2[cell]);
      const double unsold_c = exp(0.3 * lvb2) * tothi;
      for (int l = 0; l < L.nline; l++) {
        if (L.active && !L.active[l]) continue;
        const double llc = L.llam0[l] - vproj;
        const double pos = (llc - G.llam1) * G.inv_dllam;
        const int ic = (int)lround(pos) + 1;
        const int f0 = ic < 1 ? 1 : (ic > nf ? nf : ic);
        const double arg = (base + (double)L.gpref[l]) - (double)L.lower_ev[l] * ekt;
        if (arg < ex_cutoff) continue;
        double cont0, lr0, chl0;
        if (f0 == 1) { cont0 = x_lo; lr0 = lr_lo; chl0 = chl[0]; }
        else if (f0 == nf) { cont0 = x_hi; lr0 = lr_hi; chl0 = chl[nf - 1]; }
        else {
          cont0 = point_xhat64(chi_c, T, nu[f0 - 1]);
          lr0 = cont0 > 0.0 ? lt + log(cont0) : -DBL_MAX;
          if constexpr (NF > 0) {
            chl0 = chl[0];
#pragma unroll
            for (int k = 1; k < NF; k++) chl0 = (k == f0 - 1) ? chl[k] : chl0;
          } else {
            chl0 = chl[f0 - 1];
          }
        }
        double refl = tol * cont0, lref;
        const double flo = flo_scale * chl0;
        if (flo > refl) { refl = flo; lref = log(flo * sqrt_pi); }
        else lref = lr0;
        if (arg <= lref) continue;
        const double Rij = exp(arg);
        if (voigt_peak * Rij <= refl) continue;
        double a = (double)L.grad[l];
        const double gw1 = L.gw1[l];
        if (L.unsold[l]) a = fma(gw1, unsold_c, a);
        else if (gw1 != 0.0) a = fma(gw1 * exp((double)L.gw2[l] * lvb2), tothi, a);
        const double gs = L.gstk[l];
        a = gs >= 0.0 ? fma(gs, ne, a) : fma(-gs, starkpe, a);
        a *= sdl;
        const double S = Rij * D;
        const double x1 = (G.llam[f0 - 1] - llc) * G.inv_dllam;
        const QlgCoef64 cf = qlg_setup64(a, D, SQ, S);
        const double hw = qlg_halfwidth64(D2, a, S, refl, arg - lref);
        const int noff = (int)lround(fmin(hw, (double)(nf + abs(ic))));
        const int fa = ic - noff > 1 ? ic - noff : 1;
        const int fb = ic + noff < nf ? ic + noff : nf;
        if (fa > fb) continue;
        const double x0 = x1 - (double)(f0 - fa);
        if constexpr (NF > 0) {
#pragma unroll
          for (int f = 0; f < NF; f++)
            if (f + 1 >= fa && f + 1 <= fb) chl[f] += qlg_eval64(tab, cf, x0 + (double)(f + 1 - fa));
        } else {
          for (int f = fa - 1; f < fb; f++) chl[f] += qlg_eval64(tab, cf, x0 + (double)(f + 1 - fa));
        }
      }
    }
    // epilogue: transfer units (in place over the accumulator row when NF = 0)
#pragma unroll
    for (int f = 0; f < nf; f++) {
      double c, sv;
      point_units(chi_c, T, nu[f], chl[f], chl[f], (double)A.maser_chi_floor, c, sv);
      co[f] = c;
      so[f] = sv;
    }
  }
}

// max |vproj| of one ray over the cells, vproj formed as the opacity kernels form it
__global__ void k_vproj_absmax(AtmosDev A, double v0, double v1, double v2, unsigned *out) {
  unsigned m = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.ncell; c += gridDim.x * blockDim.x) {
    const float vp = (float)((v0 * (double)A.vx[c] + v1 * (double)A.vy[c]) + v2 * (double)A.vz[c]);
    m = max(m, __float_as_uint(fabsf(vp)));
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// rotate_array's weights of one plane for the fused sweep, with the periodic
// offsets already reduced to [0, n): ux = modulo(up1, nx), uy = modulo(up2, ny)
struct RotCol { int ux, uy; float a, b, c, d; };

// The four raw taps of one plane (chi and Snu), loaded ahead of their use
struct Taps { float c11, c21, c12, c22, s11, s21, s12, s22; };

__device__ __forceinline__ Taps load_taps(const float *chi, const float *S, size_t plane_off, const RotCol &r, int f,
                                          int x, int y, int nf, int nx, int ny) {
  int x1 = x + r.ux;
  x1 = x1 >= nx ? x1 - nx : x1;
  const int x2 = x1 + 1 == nx ? 0 : x1 + 1;
  int y1 = y + r.uy;
  y1 = y1 >= ny ? y1 - ny : y1;
  const int y2 = y1 + 1 == ny ? 0 : y1 + 1;
  const unsigned rx1 = (unsigned)nf * x1, rx2 = (unsigned)nf * x2;
  const unsigned ry1 = (unsigned)nf * nx * y1, ry2 = (unsigned)nf * nx * y2;
  const float *pc = chi + plane_off + f, *ps = S + plane_off + f;
  Taps t;
  t.c11 = __ldg(pc + rx1 + ry1); t.c21 = __ldg(pc + rx2 + ry1);
  t.c12 = __ldg(pc + rx1 + ry2); t.c22 = __ldg(pc + rx2 + ry2);
  t.s11 = __ldg(ps + rx1 + ry1); t.s21 = __ldg(ps + rx2 + ry1);
  t.s12 = __ldg(ps + rx1 + ry2); t.s22 = __ldg(ps + rx2 + ry2);
  return t;
}

// shifted = a p11; then b p21, c p12, d p22 added in that order (rt_patch_mod.f90:3850-3853)
__device__ __forceinline__ void combine(const Taps &t, const RotCol &r, float &xv, float &sv) {
  float v = r.a * t.c11;
  v = fmaf(r.b, t.c21, v);
  v = fmaf(r.c, t.c12, v);
  xv = fmaf(r.d, t.c22, v);
  float w = r.a * t.s11;
  w = fmaf(r.b, t.s21, w);
  w = fmaf(r.c, t.s12, w);
  sv = fmaf(r.d, t.s22, w);
}

// chi, S: (nf, nx, ny, nz) unrotated transfer units of the whole column; rot: per
// global plane; slab_z0: first global plane of each slab (nslab + 1 entries).
__global__ void __launch_bounds__(256) k_quad_rot_column(int nf, int nx, int ny, int nz, const float *chi,
                                                         const float *S, const RotCol *rot, const int *slab_z0,
                                                         int nslab, QuadConst qc, PchipConst pc, float dtmax,
                                                         float Imax, float *I_top) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t plane = (size_t)nf * nx * ny;
  if (g >= plane) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  // PCHIP ghost below the bottom slab from its unrotated planes 1 and 2
  float gx, gs, gI;
  {
    float y1 = chi[g], y2 = chi[g + plane];
    float dydx1 = (2.0f * (y2 - y1)) / pc.dx1 - 0.0f;
    gx = fmaxf((pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * dydx1 + pc.cm1 * 0.0f), 0.0f);
    y1 = S[g]; y2 = S[g + plane];
    dydx1 = (2.0f * (y2 - y1)) / pc.dx1 - 0.0f;
    gs = fmaxf((pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * dydx1 + pc.cm1 * 0.0f), 0.0f);
    gI = gs;
  }
  for (int s = 0; s < nslab; s++) {
    const int z0 = slab_z0[s], n = slab_z0[s + 1] - z0;
    float xu = gx, su = gs, Iu = gI, xc, sc, xd, sd;
    RotCol r0 = rot[z0], r1 = rot[z0 + 1];
    Taps t0 = load_taps(chi, S, plane * z0, r0, f, x, y, nf, nx, ny);
    Taps t1 = load_taps(chi, S, plane * (z0 + 1), r1, f, x, y, nf, nx, ny);
    combine(t0, r0, xc, sc);
    combine(t1, r1, xd, sd);
    for (int zl = 1; zl < n; zl++) {
      // the plane after next, loaded while this step computes
      const bool more = zl + 1 < n;
      RotCol rn;
      Taps tn;
      if (more) {
        rn = rot[z0 + zl + 1];
        tn = load_taps(chi, S, plane * (z0 + zl + 1), rn, f, x, y, nf, nx, ny);
      }
      float Inu, pl;
      quad_step<float>(xu, xc, xd, su, sc, sd, Iu, true, qc.rdsup, qc.dsup1, qc.dsup2, dtmax, Imax, false, Inu, pl);
      Iu = Inu;
      if (more) {
        xu = xc; su = sc; xc = xd; sc = sd;
        combine(tn, rn, xd, sd);
      }
    }
    float In, pl;
    quad_step<float>(xu, xc, xd, su, sc, sd, Iu, false, qc.rdsup, qc.dsup1, qc.dsup2, dtmax, Imax, false, In, pl);
    gx = xd; gs = sd; gI = In;
  }
  I_top[g] = gI;
}

// The same sweep with two neighbouring frequencies per thread (nf even): every tap
// is one 8-byte load of a frequency pair, so the sheared plane's index arithmetic
// and the loads serve two points; the rotation weights of the ray's planes sit in
// shared memory; the taps are loaded two planes ahead of their use; and the
// extinction slope t3 of a step is carried into the next step's t1 (same operands,
// same rounding).  Bit-identical to k_quad_rot_column.
struct Taps2 { float2 c11, c21, c12, c22, s11, s21, s12, s22; };

__device__ __forceinline__ Taps2 load_taps2(const float2 *chi, const float2 *S, size_t plane_off, const RotCol &r,
                                            int f2, int x, int y, int nf2, int nx, int ny) {
  int x1 = x + r.ux;
  x1 = x1 >= nx ? x1 - nx : x1;
  const int x2 = x1 + 1 == nx ? 0 : x1 + 1;
  int y1 = y + r.uy;
  y1 = y1 >= ny ? y1 - ny : y1;
  const int y2 = y1 + 1 == ny ? 0 : y1 + 1;
  const unsigned rx1 = (unsigned)nf2 * x1, rx2 = (unsigned)nf2 * x2;
  const unsigned ry1 = (unsigned)nf2 * nx * y1, ry2 = (unsigned)nf2 * nx * y2;
  const float2 *pc = chi + plane_off + f2, *ps = S + plane_off + f2;
  Taps2 t;
  t.c11 = __ldg(pc + rx1 + ry1); t.c21 = __ldg(pc + rx2 + ry1);
  t.c12 = __ldg(pc + rx1 + ry2); t.c22 = __ldg(pc + rx2 + ry2);
  t.s11 = __ldg(ps + rx1 + ry1); t.s21 = __ldg(ps + rx2 + ry1);
  t.s12 = __ldg(ps + rx1 + ry2); t.s22 = __ldg(ps + rx2 + ry2);
  return t;
}

__device__ __forceinline__ float bilin(const RotCol &r, float p11, float p21, float p12, float p22) {
  float v = r.a * p11;
  v = fmaf(r.b, p21, v);
  v = fmaf(r.c, p12, v);
  return fmaf(r.d, p22, v);
}

__device__ __forceinline__ void combine2(const Taps2 &t, const RotCol &r, float2 &xv, float2 &sv) {
  xv.x = bilin(r, t.c11.x, t.c21.x, t.c12.x, t.c22.x);
  xv.y = bilin(r, t.c11.y, t.c21.y, t.c12.y, t.c22.y);
  sv.x = bilin(r, t.s11.x, t.s21.x, t.s12.x, t.s22.x);
  sv.y = bilin(r, t.s11.y, t.s21.y, t.s12.y, t.s22.y);
}

__device__ __forceinline__ float pchip_ghost(float y1, float y2, const PchipConst &pc) {
  const float dydx1 = (2.0f * (y2 - y1)) / pc.dx1 - 0.0f;
  return fmaxf((pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * dydx1 + pc.cm1 * 0.0f), 0.0f);
}

// shared memory: the ray's RotCol of every global plane (nz entries).  Three blocks
// per SM (79 registers, no spills) measured 11 % faster than the unbounded 97.
__global__ void __launch_bounds__(256, 3) k_quad_rot_column2(int nf, int nx, int ny, int nz, const float *chi,
                                                          const float *S, const RotCol *rot, const int *slab_z0,
                                                          int nslab, QuadConst qc, PchipConst pc, float dtmax,
                                                          float Imax, float *I_top) {
  extern __shared__ RotCol s_rot[];
  for (int i = threadIdx.x; i < nz; i += blockDim.x) s_rot[i] = rot[i];
  __syncthreads();
  const int nf2 = nf >> 1;
  const size_t plane = (size_t)nf2 * nx * ny;  // in frequency pairs
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= plane) return;
  const int f2 = (int)(g % nf2), x = (int)((g / nf2) % nx), y = (int)(g / ((size_t)nf2 * nx));
  const float2 *chi2 = reinterpret_cast<const float2 *>(chi), *S2 = reinterpret_cast<const float2 *>(S);
  const float rdsup = qc.rdsup, dsup1 = qc.dsup1, dsup2 = qc.dsup2;
  // PCHIP ghost below the bottom slab from its unrotated planes 1 and 2
  float2 gx, gs, gI;
  {
    const float2 c1 = chi2[g], c2 = chi2[g + plane], s1 = S2[g], s2 = S2[g + plane];
    gx = make_float2(pchip_ghost(c1.x, c2.x, pc), pchip_ghost(c1.y, c2.y, pc));
    gs = make_float2(pchip_ghost(s1.x, s2.x, pc), pchip_ghost(s1.y, s2.y, pc));
    gI = gs;
  }
  for (int s = 0; s < nslab; s++) {
    const int z0 = slab_z0[s], n = slab_z0[s + 1] - z0;
    float2 xu = gx, su = gs, Iu = gI, xc, sc, xd, sd;
    {
      const RotCol r0 = s_rot[z0], r1 = s_rot[z0 + 1];
      const Taps2 t0 = load_taps2(chi2, S2, plane * z0, r0, f2, x, y, nf2, nx, ny);
      const Taps2 t1 = load_taps2(chi2, S2, plane * (z0 + 1), r1, f2, x, y, nf2, nx, ny);
      combine2(t0, r0, xc, sc);
      combine2(t1, r1, xd, sd);
    }
    Taps2 tn;
    RotCol rn;
    if (n > 2) {
      rn = s_rot[z0 + 2];
      tn = load_taps2(chi2, S2, plane * (z0 + 2), rn, f2, x, y, nf2, nx, ny);
    }
    float2 t1 = make_float2((xc.x - xu.x) * rdsup, (xc.y - xu.y) * rdsup);
    for (int zl = 1; zl < n; zl++) {
      // the plane two ahead, loaded while this step computes
      Taps2 tnn;
      RotCol rnn;
      if (zl + 2 < n) {
        rnn = s_rot[z0 + zl + 2];
        tnn = load_taps2(chi2, S2, plane * (z0 + zl + 2), rnn, f2, x, y, nf2, nx, ny);
      }
      const float2 t3 = make_float2((xd.x - xc.x) * rdsup, (xd.y - xc.y) * rdsup);
      float2 In;
      float pl;
      quad_step_t13<float>(t1.x, t3.x, xu.x, xc.x, xd.x, su.x, sc.x, sd.x, Iu.x, true, dsup1, dsup2, dtmax, Imax,
                           false, In.x, pl);
      quad_step_t13<float>(t1.y, t3.y, xu.y, xc.y, xd.y, su.y, sc.y, sd.y, Iu.y, true, dsup1, dsup2, dtmax, Imax,
                           false, In.y, pl);
      Iu = In;
      if (zl + 1 < n) {
        t1 = t3;
        xu = xc; su = sc; xc = xd; sc = sd;
        combine2(tn, rn, xd, sd);
        tn = tnn;
        rn = rnn;
      }
    }
    float2 In;
    float pl;
    quad_step<float>(xu.x, xc.x, xd.x, su.x, sc.x, sd.x, Iu.x, false, rdsup, dsup1, dsup2, dtmax, Imax, false, In.x,
                     pl);
    quad_step<float>(xu.y, xc.y, xd.y, su.y, sc.y, sd.y, Iu.y, false, rdsup, dsup1, dsup2, dtmax, Imax, false, In.y,
                     pl);
    gx = xd; gs = sd; gI = In;
  }
  reinterpret_cast<float2 *>(I_top)[g] = gI;
}

// save_intensity (rt_patch_mod.f90:4151-4208): ie(f) = <2h nu^5/(c^3 AA) I>_xy, in
// two deterministic stages: blocks (32 frequencies x 8 rows) sum a fixed stride of
// columns into partials, then one thread per frequency adds the partials in order.
template <typename TI>
__global__ void k_save_partial(int nf, int ncol, const double *nu, const TI *I_top, double *part) {
  __shared__ double acc[8][33];
  const int f = blockIdx.x * 32 + threadIdx.x;
  const int nparts = gridDim.y;
  double s = 0.0;
  if (f < nf) {
    const double conv = 2.0 * 6.626176e-27 / (2.99792458e10 * 2.99792458e10 * 2.99792458e10 * 1e8);
    const double n5 = nu[f] * nu[f] * nu[f] * nu[f] * nu[f];
    for (int c = blockIdx.y * blockDim.y + threadIdx.y; c < ncol; c += nparts * blockDim.y)
      s += (double)(float)(conv * n5 * (double)I_top[(size_t)f + (size_t)nf * c]);
  }
  acc[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && f < nf) {
    double t = 0.0;
    for (int k = 0; k < (int)blockDim.y; k++) t += acc[k][threadIdx.x];
    part[(size_t)blockIdx.y * nf + f] = t;
  }
}

__global__ void k_save_final(int nf, int ncol, int nparts, const double *part, float *ie) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double t = 0.0;
  for (int p = 0; p < nparts; p++) t += part[(size_t)p * nf + f];
  ie[f] = (float)t / (float)ncol;
}

// copy the transfer units of a slab's planes into its FP64 work array (plain path)
__global__ void k_slab_in(size_t plane, int n, const double *chi, const double *S, double *work, int nzs) {
  const size_t tot = plane * n;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < tot; g += (size_t)gridDim.x * blockDim.x) {
    work[g + plane] = chi[g];
    work[g + plane + plane * (nzs + 2)] = S[g];
  }
}

}  // namespace m3d

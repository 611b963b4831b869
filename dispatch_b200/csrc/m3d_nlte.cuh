// Model-atom opacities and ALI rate integrals of one frequency window
// (non-hydrogen lines), FP32 with the reference's real(8) constants:
//   bound_bound_damping / line_damping    SRC/rt_patch_mod.f90:2649-2681, HOP/bbtrans_mod.f90:78-106
//   add_bound_free_opacities              SRC/rt_patch_mod.f90:2581-2643
//   foreground's split start              SRC/rt_patch_mod.f90:1474-1487
//   add_bound_bound_opacities             SRC/rt_patch_mod.f90:2689-2831
//   add_largest / other_contribution      SRC/rt_patch_mod.f90:3150-3187
//   work_to_transfer_units (split form)   SRC/rt_patch_mod.f90:3571-3651
//   bound_bound_rates                     SRC/rt_patch_mod.f90:2852-3142
//   bound_free_rates                      SRC/rt_patch_mod.f90:3193-3259
//   integrate_rates                       SRC/rt_patch_mod.f90:3437-3465
//   normalize_profiles                    SRC/atom_mod.f90:377-430
//   combine_twin_hemispheres' average     SRC/rt_patch_mod.f90:1812-1887
//
// The opacity kernels give one thread one (f, cell) point, which walks the
// transitions that cover f in their window order, so every point accumulates
// in the reference's order.  The rate kernels give one thread one
// (transition, cell) pair, which sums over the transition's points in f
// order.  A real(4) local assigned from a real(8) expression is rounded where
// the Fortran assigns it.
#pragma once
#include "m3d_qlg.cuh"

namespace m3d {

struct NlWinDev {
  int nf, nline, ncont;
  const int *li, *lj, *lntrans, *lindex, *lblue, *lred, *loff;
  const float *q;
  const double *wnu, *wq, *Bij, *Aij, *lower_ev, *grad, *gw1, *gw2, *gstk;
  const unsigned char *lactive, *lsums, *unsold;
  const int *ci, *cj, *cntrans, *cblue, *cred, *coff;
  const float *alpha;
  const double *cwnu;
  const unsigned char *cactive;
  const double *g, *ev;
  double cut_x;
  // per frequency: the active lines / continua whose window holds f, ascending
  const int *lf_ptr, *lf_idx, *cf_ptr, *cf_idx;
};

// qlg_bot_profile (qlg_mod.f90:682-689)
__device__ __forceinline__ float nl_profile(const float2 *tab, float a, float q, float vpr, float idf) {
  const float v = fabsf(q - vpr) * idf;
  const QlgCoef c = qlg_setup(a, 1.0f, 0.8325546112f, 1.7724538509f);
  // the reciprocal of 1 + (v ih)^2 by rcp_markstein where the converged lanes all
  // keep it below 2^126 (v ih <= 2^62), else by __frcp_rn: the same bits either way
  const bool mk = __all_sync(__activemask(), v * c.ih <= 4611686018427387904.0f);
  const float K1 = mk ? qlg_eval<true>(tab, c, v) : qlg_eval<false>(tab, c, v);
  return ((K1 * 0.5641895835f) * idf) * (q + 1.0f);
}

__global__ void k_bb_damping(NlWinDev W, int ncell, const float *__restrict__ ne, const float *__restrict__ tothi,
                             const float *__restrict__ vbar2, const float *__restrict__ stark_pe,
                             const float *__restrict__ unsold, const float *__restrict__ inv_df,
                             float *__restrict__ adamp) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    for (int i = 0; i < W.nline; i++) {
      if (W.lactive && !W.lactive[i]) continue;
      float a = 0.0f;
      if (W.unsold[i]) a = (float)((double)a + W.gw1[i] * (double)unsold[c]);
      else a = (float)((double)a + (W.gw1[i] == 0.0 ? 0.0 : W.gw1[i] * pow((double)vbar2[c], W.gw2[i]) * (double)tothi[c]));
      if (W.gstk[i] >= 0.0) a = (float)((double)a + W.gstk[i] * (double)ne[c]);
      else a = (float)((double)a - W.gstk[i] * (double)stark_pe[c]);
      a = (float)((double)a + W.grad[i]);
      adamp[(size_t)c + (size_t)ncell * i] = a * inv_df[c];
    }
  }
}

__global__ void k_bf_opacity(NlWinDev W, int ncell, const double *__restrict__ b, const double *__restrict__ nstar,
                             const double *__restrict__ pop_ratio, const double *__restrict__ e_kT,
                             float *__restrict__ xhat, float *__restrict__ ehat) {
  const size_t nf = (size_t)W.nf, n = nf * ncell;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(k % nf), c = (int)(k / nf);
    const int p0 = W.cf_ptr[f], p1 = W.cf_ptr[f + 1];
    if (p0 == p1) continue;
    float xh = xhat[k], eh = ehat[k];
    for (int p = p0; p < p1; p++) {
      const int i = W.cf_idx[p];
      const int li = W.ci[i], lj = W.cj[i];
      const double ns = nstar[(size_t)c + (size_t)ncell * li];
      float ni, tmp;
      if (b) {
        ni = (float)(ns * b[(size_t)c + (size_t)ncell * li] * pop_ratio[c]);
        tmp = (float)(ns * b[(size_t)c + (size_t)ncell * lj] * pop_ratio[c]);
        if ((W.ev[lj] - W.ev[li]) * e_kT[c] > W.cut_x) tmp = 0.0f;
      } else {
        ni = (float)(ns * pop_ratio[c]);
        tmp = ni;
      }
      const float alpha = W.alpha[W.coff[i] + f - W.cblue[i]];
      xh = xh + alpha * ni;
      eh = eh + alpha * tmp;
    }
    xhat[k] = xh;
    ehat[k] = eh;
  }
}

__device__ __forceinline__ void add_largest(float value, int index, float &largest, float &rest, int &largest_index) {
  if (fabsf(value) > fabsf(largest)) {
    rest = rest + largest;
    largest = value;
    largest_index = index;
  } else {
    rest = rest + value;
  }
}

__device__ __forceinline__ float other_contribution(float value, int index, float largest, float rest,
                                                    int largest_index) {
  return index == largest_index ? rest : largest + (rest - value);
}

// work_to_transfer_units of one point with split rates: (xhat, L, R) -> (chi, S)
__device__ __forceinline__ bool units_split_point(float xhat, float be, float sL, float sR, float sc, bool has_scat,
                                                  float fl, int suppress, float &chi_out, float &S_out) {
  const float eta_rest = be * sR;
  float eta = be * sL + eta_rest;
  float chi = xhat - eta;
  if (has_scat) eta = be * sL + (eta_rest + sc);
  const float floor_ = fmaxf(fl * fabsf(xhat), FLT_MIN);
  bool floored = false;
  if (suppress) chi = fmaxf(chi, floor_);
  else if (fabsf(chi) < floor_) { chi = copysignf(floor_, chi); floored = true; }
  chi_out = chi;
  S_out = eta / chi;
  return floored;
}

struct NlSplit {
  float *sopL, *sopR, *schL, *schR;
  int *sid, *schid;
};

__global__ void k_bb_opacity(NlWinDev W, int ncell, const double *__restrict__ b, const double *__restrict__ nstar,
                             const double *__restrict__ pop_ratio, const double *__restrict__ e_kT,
                             const float *__restrict__ inv_df, const float *__restrict__ vproj,
                             const float *__restrict__ adamp, const float2 *__restrict__ tab, int lte,
                             float *__restrict__ xhat, float *__restrict__ ehat, NlSplit S,
                             const float *__restrict__ units_beta = nullptr, float units_floor = 0.0f,
                             const float *__restrict__ xin = nullptr, const float *__restrict__ ein = nullptr) {
  const size_t nf = (size_t)W.nf, n = nf * ncell;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(k % nf), c = (int)(k / nf);
    // the background from xin/ein where given (xhat/ehat then only receive the result)
    float xh = xin ? xin[k] : xhat[k], eh = ein ? ein[k] : ehat[k];
    float oL = eh, oR = 0.0f, cL = xh, cR = 0.0f;
    int oid = 0, cid = 0;
    const int p0 = W.lf_ptr[f], p1 = W.lf_ptr[f + 1];
    if (p0 < p1) {
      const float idf = inv_df[c], vpr = vproj[c], ekt = (float)e_kT[c];
      for (int p = p0; p < p1; p++) {
        const int i = W.lf_idx[p];
        const int li = W.li[i], lj = W.lj[i];
        const float ni = (float)(nstar[(size_t)c + (size_t)ncell * li] * pop_ratio[c]);
        float bi = 1.0f, bj = 1.0f;
        if (!lte && b) {
          bi = (float)b[(size_t)c + (size_t)ncell * li];
          bj = (float)b[(size_t)c + (size_t)ncell * lj];
        }
        const float lower_off = (float)(W.lower_ev[i] - W.ev[li]);
        if (lower_off != 0.0f) {
          bi = bi * expf(-lower_off * ekt);
          bj = bj * expf(-lower_off * ekt);
        }
        const float phi = nl_profile(tab, adamp[(size_t)c + (size_t)ncell * i], W.q[W.loff[i] + f - W.lblue[i]], vpr, idf);
        const float Rij = (float)((double)ni * W.Bij[i]);
        const float eta_fac = Rij * bj, chi_fac = Rij * bi;
        xh = xh + phi * chi_fac;
        eh = eh + phi * eta_fac;
        if (S.sopL) {
          add_largest(phi * eta_fac, W.lindex[i], oL, oR, oid);
          add_largest(phi * chi_fac, W.lindex[i], cL, cR, cid);
        }
      }
      if (!units_beta) {
        xhat[k] = xh;
        ehat[k] = eh;
      }
    }
    // fused work_to_transfer_units (split form, no scattering term, masers floored):
    // every point leaves as chi and S
    if (units_beta) {
      float chi, Sv;
      units_split_point(xh, units_beta[k], oL, oR, 0.0f, false, units_floor, 0, chi, Sv);
      xhat[k] = chi;
      ehat[k] = Sv;
    }
    if (S.sopL) {
      S.sopL[k] = oL;
      S.sopR[k] = oR;
      S.sid[k] = oid;
      S.schL[k] = cL;
      S.schR[k] = cR;
      S.schid[k] = cid;
    }
  }
}

// the direction's profile integral of the lines that sum over windows, one
// thread per (line, cell): wphi(cell, ntrans) += wmu * sum(phi * wq)
__global__ void k_bb_wphi(NlWinDev W, int ncell, const float *__restrict__ inv_df, const float *__restrict__ vproj,
                          const float *__restrict__ adamp, const float2 *__restrict__ tab, float wmu,
                          float *__restrict__ wphi) {
  const size_t n = (size_t)ncell * W.nline;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(k % ncell), i = (int)(k / ncell);
    if ((W.lactive && !W.lactive[i]) || !W.lsums[i]) continue;
    const float idf = inv_df[c], vpr = vproj[c], a = adamp[k];
    double s = 0.0;
    for (int f = W.lblue[i]; f <= W.lred[i]; f++) {
      const int o = W.loff[i] + f - W.lblue[i];
      s = s + (double)nl_profile(tab, a, W.q[o], vpr, idf) * W.wq[o];
    }
    const size_t kw = (size_t)c + (size_t)ncell * W.lntrans[i];
    wphi[kw] = wphi[kw] + wmu * (float)s;
  }
}

__global__ void k_transfer_units_split(size_t n, float *__restrict__ w1, float *__restrict__ w2,
                                       const float *__restrict__ beta, const float *__restrict__ sopL,
                                       const float *__restrict__ sopR, const float *__restrict__ scat, float fl,
                                       int suppress, int *n_floored) {
  int cnt = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    float chi, S;
    cnt += units_split_point(w1[k], beta[k], sopL[k], sopR[k], scat ? scat[k] : 0.0f, scat != nullptr, fl,
                             suppress, chi, S);
    w1[k] = chi;
    w2[k] = S;
  }
  if (n_floored && cnt) atomicAdd(n_floored, cnt);
}

struct NlRateOpts { int split, precond, per_direction, use_flags, do_scat; float wmu, wtot; };

struct NlRadField {
  const float *work1, *inu, *psi, *irem, *escape, *beta, *Bnu, *scat;
  const float *sopL, *sopR, *schL, *schR;
  const int *sid, *schid;
};

// Both rate kernels give one warp to one (cell, transition): its lanes evaluate
// the window's frequencies 32 at a time, reading the per-point arrays along f
// (coalesced), and lanes 0..3 then add the terms in ascending f out of shared
// memory, so that every sum keeps the reference's left-to-right order.
constexpr int kRateWarps = 8;

__device__ __forceinline__ void rate_chunk_sum(float (*T)[33], int lane, int cnt, float &acc) {
  __syncwarp();
  if (lane < 4)
    for (int j = 0; j < cnt; j++) acc = acc + T[lane][j];
  __syncwarp();
}

// bound_bound_rates: one warp per (line, kBbCells consecutive cells).  The first
// kBbCells lanes form their cell's per-line constants; the terms of every (cell, f) are then evaluated
// a cell at a time with all 32 lanes along f (one 128-byte load per array), written
// to shared memory, and lane k adds cell k's terms in ascending f -- the
// reference's order.  A line window of up to 32 points takes a single chunk.
// The tiles run cell-major: the lines of a tile's cells are neighbouring warps, so the
// sectors their windows share (and those a window straddles) are read from DRAM
// once and from L2 after.  Each (line, cell) has one writer, so the order changes
// no sum.
// 8 cells a tile (17 KB of shared terms a block) and 64 registers give 8 blocks (32
// warps) per SM, which hides the loads' latency better than 16-cell tiles at 6 blocks:
// the 120^3 window's sweep 748 -> 711 ms
constexpr int kBbWarps = 4, kBbCells = 8;

__global__ void __launch_bounds__(kBbWarps * 32, 8)
k_bb_rates(NlWinDev W, NlRateOpts O, int ncell, const double *__restrict__ b,
           const double *__restrict__ nstar, const double *__restrict__ pop_ratio,
           const double *__restrict__ e_kT, const float *__restrict__ inv_df,
           const float *__restrict__ vproj, const float *__restrict__ adamp,
           const float2 *__restrict__ tab, NlRadField R, const unsigned *__restrict__ flags_in,
           unsigned *__restrict__ flags_raise, float *__restrict__ gamma_ij,
           float *__restrict__ gamma_ji) {
  __shared__ float sh[kBbWarps][4][kBbCells][33];
  __shared__ int shr[kBbWarps][kBbCells];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float (*T)[kBbCells][33] = sh[wib];
  const size_t nf = (size_t)W.nf;
  const int ctiles = (ncell + kBbCells - 1) / kBbCells;
  const size_t ntile = (size_t)ctiles * W.nline;
  const size_t stride = (size_t)gridDim.x * kBbWarps;
  for (size_t tt = (size_t)blockIdx.x * kBbWarps + wib; tt < ntile; tt += stride) {
    const int i = (int)(tt % W.nline), c0 = (int)(tt / W.nline) * kBbCells;
    if (W.lactive && !W.lactive[i]) continue;
    const int li = W.li[i], lj = W.lj[i], fs = W.lblue[i], fe = W.lred[i], off = W.loff[i];
    const bool own_norm = O.per_direction && !W.lsums[i];
    const int index = W.lindex[i];
    const double Aij = W.Aij[i];
    const float lower_off = (float)(W.lower_ev[i] - W.ev[li]);
    const int t = W.lntrans[i], pw = t >> 5, pb = t & 31;
    const int ncl = min(kBbCells, ncell - c0);
    // lane k < ncl: the constants of cell c0 + k for this line
    const int c = c0 + lane;
    const bool mine = lane < ncl;
    float ni = 0.0f, nj = 0.0f, inv_nref = 0.0f, eta_coef = 0.0f, abs_coef = 0.0f, g_ratio = 0.0f;
    float idf = 0.0f, vpr = 0.0f, a = 0.0f;
    int in_force = 0;
    if (mine) {
      const double nsi = nstar[(size_t)c + (size_t)ncell * li], nsj = nstar[(size_t)c + (size_t)ncell * lj];
      const double bbi = b[(size_t)c + (size_t)ncell * li], bbj = b[(size_t)c + (size_t)ncell * lj];
      ni = (float)(bbi * nsi);
      nj = (float)(bbj * nsj);
      idf = inv_df[c];
      vpr = vproj[c];
      a = adamp[(size_t)c + (size_t)ncell * i];
      const float ekt = (float)e_kT[c];
      if (nsi > 0 && nsj > 0) {
        const double beta_ref = nsj * W.g[li] / (nsi * W.g[lj]);
        inv_nref = (float)fmin((1.0 - beta_ref) / beta_ref, 1e35);
      }
      if (lower_off != 0.0f) {
        ni = ni * expf(-lower_off * ekt);
        nj = nj * expf(-lower_off * ekt);
      }
      if (O.precond) {
        float split_bj = (float)bbj;
        if (lower_off != 0.0f) split_bj = split_bj * expf(-lower_off * ekt);
        float split_Rij = (float)(nsi * pop_ratio[c]);
        split_Rij = (float)((double)split_Rij * W.Bij[i]);
        eta_coef = split_Rij * split_bj;
        float split_bi = (float)bbi;
        if (lower_off != 0.0f) split_bi = split_bi * expf(-lower_off * ekt);
        abs_coef = split_Rij * split_bi;
        if (nj > 0.0f) g_ratio = (float)((double)(ni / nj) * (W.g[lj] / W.g[li]));
      }
      if (O.split && O.precond && O.use_flags) in_force = (flags_in[(size_t)c + (size_t)ncell * pw] >> pb) & 1u;
    }
    if (lane < kBbCells) shr[wib][lane] = 0;
    __syncwarp();
    // lane k < 16 accumulates sums (A, I, P, w) without the split, (T, U, -, w) with it, of cell c0 + k
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
    for (int f0 = fs; f0 <= fe; f0 += 32) {
      const int f = f0 + lane;
      const int o = off + f - fs;
      const bool fin = f <= fe;
      float wmunu = 0.0f, wqf = 0.0f, qf = 0.0f;
      if (fin) {
        qf = W.q[o];
        wmunu = (float)((double)O.wmu * W.wnu[o] * Aij);
        wqf = (float)W.wq[o];
      }
      for (int ci = 0; ci < ncl; ci++) {
        const float c_idf = __shfl_sync(0xffffffffu, idf, ci), c_vpr = __shfl_sync(0xffffffffu, vpr, ci);
        const float c_a = __shfl_sync(0xffffffffu, a, ci), c_inr = __shfl_sync(0xffffffffu, inv_nref, ci);
        const float c_eta = __shfl_sync(0xffffffffu, eta_coef, ci), c_abs = __shfl_sync(0xffffffffu, abs_coef, ci);
        const int c_if = __shfl_sync(0xffffffffu, in_force, ci);
        float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f, t3 = 0.0f;
        if (fin) {
          const size_t k = (size_t)f + nf * (size_t)(c0 + ci);
          const float phi = nl_profile(tab, c_a, qf, c_vpr, c_idf);
          t3 = phi * wqf;
          if (!O.split) {
            const float vvv = phi * wmunu;
            t0 = vvv * (R.Bnu[k] * c_inr);
            t1 = vvv * R.inu[k];
            t2 = vvv * phi * R.psi[k] * R.beta[k];
          } else {
            const float nb = R.Bnu[k];
            const float vvv = phi * wmunu;
            if (O.precond) {
              const float be = R.beta[k];
              float psi = R.psi[k];
              const float eta_u = phi * c_eta;
              const float eta_t = eta_u * be;
              const float chi_t = phi * c_abs - eta_t;
              const float eta_other = be * other_contribution(eta_u, index, R.sopL[k], R.sopR[k], R.sid[k]);
              const float chi_other = other_contribution(phi * c_abs, index, R.schL[k], R.schR[k], R.schid[k]) - eta_other;
              float other = eta_other;
              if (O.do_scat) other = other + R.scat[k];
              if (chi_t < 0.0f || c_if) psi = 0.0f;
              if (psi == 0.0f) shr[wib][ci] = 1;
              const float up = psi == 0.0f ? R.inu[k] : R.irem[k] + psi * other;
              const float spont = psi == 0.0f ? 1.0f : (chi_other + R.escape[k] * chi_t) / R.work1[k];
              t0 = vvv * spont * (nb * c_inr);
              t1 = vvv * (up - nb * spont);
            } else {
              t0 = vvv * (nb * c_inr);
              t1 = vvv * (R.inu[k] - nb);
            }
          }
        }
        T[0][ci][lane] = t0;
        T[1][ci][lane] = t1;
        T[2][ci][lane] = t2;
        T[3][ci][lane] = t3;
      }
      __syncwarp();
      if (mine) {
        const int cnt = min(32, fe - f0 + 1);
        for (int j = 0; j < cnt; j++) {
          s0 = s0 + T[0][lane][j];
          s1 = s1 + T[1][lane][j];
          s2 = s2 + T[2][lane][j];
          s3 = s3 + T[3][lane][j];
        }
      }
      __syncwarp();
    }
    if (mine) {
      const int raise = shr[wib][lane];
      if (O.split && O.precond && O.use_flags && raise && !in_force)
        atomicOr(&flags_raise[(size_t)c + (size_t)ncell * pw], 1u << pb);
      float g_th = s0, g_dev = s1;
      if (!O.split) {
        if (O.precond) {
          g_th = g_th - s2 * eta_coef * (g_ratio - 1.0f);
          g_dev = g_dev - s2 * eta_coef;
        }
        if (inv_nref > 0.0f) g_dev = g_dev - g_th / inv_nref;
      }
      if (own_norm && s3 > 0.0f) {
        g_th = g_th / (s3 * O.wtot);
        g_dev = g_dev / (s3 * O.wtot);
      }
      const size_t kk = (size_t)c + (size_t)ncell * i;
      gamma_ij[kk] = gamma_ij[kk] + g_th;
      gamma_ji[kk] = gamma_ji[kk] + g_dev;
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kRateWarps * 32)
k_bf_rates(NlWinDev W, int ncell, int precond, const double *__restrict__ b,
           const double *__restrict__ nstar, const double *__restrict__ e_kT,
           const float *__restrict__ twohnu3_c2, const float *__restrict__ Jnu,
           const float *__restrict__ PsiJ, const float *__restrict__ beta,
           float *__restrict__ gamma_ij, float *__restrict__ gamma_ji) {
  __shared__ float sh[kRateWarps][4][33];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float (*T)[33] = sh[wib];
  const size_t nf = (size_t)W.nf, n = (size_t)ncell * W.ncont;
  const size_t stride = (size_t)gridDim.x * kRateWarps;
  for (size_t kk = (size_t)blockIdx.x * kRateWarps + wib; kk < n; kk += stride) {
    const int c = (int)(kk % ncell), j = (int)(kk / ncell);
    if (W.cactive && !W.cactive[j]) continue;
    const int li = W.ci[j], lj = W.cj[j], fs = W.cblue[j], fe = W.cred[j], off = W.coff[j];
    if ((W.ev[lj] - W.ev[li]) * e_kT[c] > W.cut_x) continue;
    // lanes 0, 1, 2 accumulate sum_abs, sum_ems, sum_pre
    float acc = 0.0f;
    for (int f0 = fs; f0 <= fe; f0 += 32) {
      const int f = f0 + lane;
      float t0 = 0.0f, t1 = 0.0f, t2 = 0.0f;
      if (f <= fe) {
        const size_t k = (size_t)f + nf * c;
        const int o = off + f - fs;
        const float wmunu = (float)(0.5 * W.cwnu[o]);
        const float vij = twohnu3_c2[f] * W.alpha[o] * wmunu;
        const float vji = vij * beta[k];
        const float phi = PsiJ[k] * W.alpha[o];
        t0 = vij * Jnu[k];
        t1 = vji * (Jnu[k] + 1.0f);
        t2 = vji * phi;
      }
      T[0][lane] = t0;
      T[1][lane] = t1;
      T[2][lane] = t2;
      T[3][lane] = 0.0f;
      rate_chunk_sum(T, lane, min(32, fe - f0 + 1), acc);
    }
    const float sum_abs = __shfl_sync(0xffffffffu, acc, 0), sum_ems = __shfl_sync(0xffffffffu, acc, 1);
    const float sum_pre = __shfl_sync(0xffffffffu, acc, 2);
    if (lane == 0) {
      float g_ij = sum_abs, g_ji = sum_ems;
      if (precond) {
        const double nsi = nstar[(size_t)c + (size_t)ncell * li];
        g_ij = (float)((double)g_ij - (double)sum_pre * nsi * b[(size_t)c + (size_t)ncell * lj]);
        g_ji = (float)((double)g_ji - (double)sum_pre * nsi * b[(size_t)c + (size_t)ncell * li]);
      }
      const size_t kg = (size_t)c + (size_t)ncell * (W.nline + j);
      gamma_ij[kg] = gamma_ij[kg] + g_ij;
      gamma_ji[kg] = gamma_ji[kg] + g_ji;
    }
  }
}

// integrate_rates: the window's sums into the atom's rates by transition index
__global__ void k_integrate_rates(NlWinDev W, int ncell, const float *__restrict__ gw_ij,
                                  const float *__restrict__ gw_ji, float *__restrict__ g_ij,
                                  float *__restrict__ g_ji) {
  const int ntr = W.nline + W.ncont;
  const size_t n = (size_t)ncell * ntr;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(k % ncell), i = (int)(k / ncell);
    const int t = i < W.nline ? W.lntrans[i] : W.cntrans[i - W.nline];
    const size_t ka = (size_t)c + (size_t)ncell * t;
    g_ij[ka] = g_ij[ka] + gw_ij[k];
    g_ji[ka] = g_ji[ka] + gw_ji[k];
  }
}

struct NlNormArgs {
  int nline, nrad, first_iter;
  const int *ti, *tj;
  const unsigned char *active, *has_wphi;
};

__global__ void k_normalize_profiles(NlNormArgs A, int ncell, const double *__restrict__ nstar,
                                     float *__restrict__ wphi, float *__restrict__ gamma_ij,
                                     float *__restrict__ gamma_ji) {
  const size_t n = (size_t)ncell * A.nrad;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(k % ncell), i = (int)(k / ncell);
    if (A.active && !A.active[i]) continue;
    if (i < A.nline) {
      if (!A.has_wphi[i]) continue;
      float w = wphi[k];
      if (A.first_iter) {
        w = w > 0.0f ? 1.0f / w : 1.0f;
        wphi[k] = w;
      }
      gamma_ij[k] = gamma_ij[k] * w;
      gamma_ji[k] = gamma_ji[k] * w;
    } else {
      gamma_ji[k] = (float)((double)gamma_ji[k] *
                            (nstar[(size_t)c + (size_t)ncell * A.ti[i]] / nstar[(size_t)c + (size_t)ncell * A.tj[i]]));
    }
  }
}

// the average of two hemispheres' J (and PsiJ), stored in both
__global__ void k_combine_twins(size_t n, float *__restrict__ a, float *__restrict__ b) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const float v = 0.5f * (a[k] + b[k]);
    a[k] = v;
    b[k] = v;
  }
}

}  // namespace m3d

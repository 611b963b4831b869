// sm_100a kernels of the radiative-transfer hot path.  Every array uses the
// reference's layout, frequency fastest, so consecutive threads own consecutive
// frequencies of one (x, y) column and every access along a sweep is coalesced.
#pragma once
#include <cstdint>

#include "m3d_math.cuh"
#include "m3d_qlg.cuh"

namespace m3d {

__device__ __forceinline__ size_t iw(int f, int x, int y, int z, int k, int nf, int nx, int ny, int nz) {
  return (size_t)f + (size_t)nf * ((size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * ((size_t)z + (size_t)(nz + 2) * (size_t)k)));
}
__device__ __forceinline__ size_t ip(int f, int x, int y, int z, int nf, int nx, int ny) {
  return (size_t)f + (size_t)nf * ((size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)(z - 1)));
}
__device__ __forceinline__ size_t ic3(int x, int y, int z, int nx, int ny) {
  return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)(z - 1));
}
__device__ __forceinline__ int wrap(int v, int n) { v %= n; return v < 0 ? v + n : v; }

constexpr double M3D_H_K = 6.626176e-27 / 1.380662e-16;  // h/k (const_mod.f90:39,43,71)

// correctly rounded reciprocal: the same value as the IEEE quotient 1/x
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }

template <typename T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }
__device__ __forceinline__ float tmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float tmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double tmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double tmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float tabs(float a) { return fabsf(a); }
__device__ __forceinline__ double tabs(double a) { return fabs(a); }
__device__ __forceinline__ float tcopysign(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ double tcopysign(double a, double b) { return copysign(a, b); }


// ----------------------------------------------------------------------------
// K0 diagnostics: the weights elementwise
// ----------------------------------------------------------------------------
__global__ void k_weights_f32(int which, int n, const float *t, float *o1, float *o2, float *o3, float *o4) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float x = t[i];
    switch (which) {
      case 0: { float E, u; exp_neg(x, E, u); o1[i] = E; o2[i] = u; } break;
      case 1: { float E, W, P, S; linear_weights(x, E, W, P, S); o1[i] = E; o2[i] = W; o3[i] = P; o4[i] = S; } break;
      case 2: { float E, U0, U1, q; parab_moments(x, E, U0, U1, q); o1[i] = E; o2[i] = U0; o3[i] = U1; o4[i] = q; } break;
      case 3: o1[i] = exp4(x); break;
      case 5: { float E; bezier3_weights(x, E, o1[i], o2[i], o3[i], o4[i]); } break;
      default: o1[i] = logf_m3d(x); break;
    }
  }
}

__global__ void k_weights_f64(int which, int n, const double *t, double *o1, double *o2, double *o3, double *o4) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = t[i];
    if (which == 1) { double E, W, P, S; linear_weights(x, E, W, P, S); o1[i] = E; o2[i] = W; o3[i] = P; o4[i] = S; }
    else { double E, U0, U1, q; parab_moments(x, E, U0, U1, q); o1[i] = E; o2[i] = U0; o3[i] = U1; o4[i] = q; }
  }
}

// qlg_bot_profile (qlg_mod.f90:682-689)
__global__ void k_qlg_profile(int n, const float2 *tab, const float *a, const float *q,
                              const float *vpr, const float *idf, float *h) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float v = fabsf(q[i] - vpr[i]) * idf[i];
    const QlgCoef c = qlg_setup(a[i], 1.0f, 0.8325546112f, 1.7724538509f);
    const float K1 = qlg_eval(tab, c, v);
    h[i] = ((K1 * 0.5641895835f) * idf[i]) * (q[i] + 1.0f);
  }
}

// ----------------------------------------------------------------------------
// Line opacity of one cell by one warp (add_opacity_equi, linelist_mod.f90:729-960)
// ----------------------------------------------------------------------------
struct LineArgs {
  int nline;
  const double *llam0;
  const float *lower_ev, *gpref, *grad, *gw1, *gw2, *gstk;
  const uint8_t *unsold;
  const int *lev_i, *lev_j;
  const uint8_t *active;
  // has_reach: the per-line reach of a previous run, and the lines select_lines
  // kept for this call (0-based, ascending; *nsel of them); null without reach
  const float *reach_in;
  const int *sel, *nsel;
};

struct GridArgs {
  int nf;
  const double *llam;
  double llam1, inv_dllam, dllam;
  float sdl, tol, flo_scale;
};

struct CellArgs {
  float idf, vbar2, ekt, ne, tothi, starkpe, vproj, base;
};

__device__ __forceinline__ float line_damping_a(const LineArgs &L, int l, float unsold_c, float lvb2,
                                                float tothi, float ne, float starkpe) {
  float a = L.grad[l];
  const float gw1 = L.gw1[l];
  // a line without van der Waals broadening adds fmaf(0*w, tothi, a) = a exactly
  // (grad >= 0, finite tothi), so the power is skipped for it
  if (L.unsold[l]) a = fmaf(gw1, unsold_c, a);
  else if (gw1 != 0.0f) a = fmaf(gw1 * exp4(L.gw2[l] * lvb2), tothi, a);
  const float gs = L.gstk[l];
  if (gs >= 0.0f) a = fmaf(gs, ne, a);
  else a = fmaf(-gs, starkpe, a);
  return a;
}

// chi, eta, cont, logref point at this cell's nf values (shared or global memory).
// dep(level) returns the departure coefficient of a 1-based level of this cell.
// diag: strength/reach/used as the reference updates them.  Lanes of the warp
// first screen 32 lines at a time against the unfloored tolerance reference and
// window (a superset of the lines the exact test keeps, since the floor only
// raises the reference), then the candidates go through the exact test in line
// order, so chi accumulates in exactly the reference's order.
template <class DepFn>
__device__ void warp_cell_lines(const LineArgs &L, const GridArgs &G, const CellArgs &c, float *chi, float *eta,
                                const float *cont, const float *logref, DepFn dep, bool do_nlte, bool diag,
                                uint8_t *used, float *strength, float *reach, const float2 *tab, int lane,
                                const float *one_m_eps = nullptr, float *chi_scat = nullptr) {
  const float ex_cutoff = -85.0f, voigt_peak = 0.5641895835f, sqrt_pi = 1.7724538509f;
  const int nf = G.nf;
  const QlgCell qw = qlg_cell(G.sdl / c.idf);
  const float lvb2 = logf_m3d(c.vbar2);
  const float unsold_c = exp4(0.3f * lvb2) * c.tothi;
  const int nline = L.sel ? *L.nsel : L.nline;
  const double lam_lo = G.llam[0], lam_hi = G.llam[nf - 1];
  for (int l0 = 0; l0 < nline; l0 += 32) {
    const int l = l0 + lane < nline ? (L.sel ? L.sel[l0 + lane] : l0 + lane) : -1;
    bool cand = false;
    if (l >= 0 && (L.active == nullptr || L.active[l])) {
      const double llc = L.llam0[l] - (double)c.vproj;
      const double pos = (llc - G.llam1) * G.inv_dllam;
      const int ic = (int)lround(pos) + 1;
      const int f0 = ic < 1 ? 1 : (ic > nf ? nf : ic);
      const float ex = L.lower_ev[l] * c.ekt;
      const float arg = (c.base + L.gpref[l]) - ex;
      const bool outside = L.reach_in && (llc < lam_lo || llc > lam_hi);
      if (!(arg < ex_cutoff) && outside) {
        // centred beyond the chunk: its exact test is arg > logref at the nearer end
        cand = arg > logref[f0 - 1] - 1e-3f;
      } else if (!(arg < ex_cutoff)) {
        const float lr = logref[f0 - 1];
        if (arg > lr - 1e-3f) {
          const float Rij = exp4(arg);
          const float ref0 = G.tol * cont[f0 - 1];
          if (voigt_peak * Rij > ref0) {
            if (diag) {
              cand = true;
            } else {
              const float a = line_damping_a(L, l, unsold_c, lvb2, c.tothi, c.ne, c.starkpe) * G.sdl;
              const float hw = qlg_halfwidth(qw, a, Rij * qw.D, ref0, (arg - lr) + 1e-3f);
              const int noff = (int)lroundf(fminf(fmaf(hw, 1.001f, 1.0f), (float)(nf + abs(ic))));
              cand = (ic - noff <= nf) && (ic + noff >= 1);
            }
          }
        }
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, cand);
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      const int ln = L.sel ? L.sel[l0 + j] : l0 + j;
      const double llc = L.llam0[ln] - (double)c.vproj;
      const double pos = (llc - G.llam1) * G.inv_dllam;
      const int ic = (int)lround(pos) + 1;
      const int f0 = ic < 1 ? 1 : (ic > nf ? nf : ic);
      const float ex = L.lower_ev[ln] * c.ekt;
      const float arg = (c.base + L.gpref[ln]) - ex;
      const bool outside = L.reach_in && (llc < lam_lo || llc > lam_hi);
      float refl, lref, cap = FLT_MAX;
      if (outside) {
        // f0 is the nearer chunk end here; no floor, no peak test, window capped by the reach
        lref = logref[f0 - 1];
        if (arg <= lref) continue;
        refl = G.tol * cont[f0 - 1];
        cap = (float)((double)L.reach_in[ln] * G.inv_dllam);
      } else {
        refl = G.tol * cont[f0 - 1];
        const float flo = G.flo_scale * chi[f0 - 1];
        if (flo > refl) { refl = flo; lref = logf_m3d(flo * sqrt_pi); }
        else lref = logref[f0 - 1];
        if (arg <= lref) continue;
      }
      const float Rij = exp4(arg);
      if (!outside && voigt_peak * Rij <= refl) continue;
      float bi = 1.0f, bj = 1.0f;
      const bool nlte_line = do_nlte && L.lev_i && L.lev_j && L.lev_i[ln] > 0 && L.lev_j[ln] > 0;
      if (nlte_line) {
        bi = dep(L.lev_i[ln]);
        bj = dep(L.lev_j[ln]);
      }
      const float a = line_damping_a(L, ln, unsold_c, lvb2, c.tothi, c.ne, c.starkpe) * G.sdl;
      if (diag && lane == 0 && !outside) {
        const float st = (voigt_peak * Rij) / cont[f0 - 1];
        atomicMax(reinterpret_cast<int *>(strength + ln), __float_as_int(st));
      }
      const float lnq = arg - lref;
      // qlg_bot_line_sweep (qlg_mod.f90:646-671)
      const float S = Rij * qw.D;
      const int i1 = f0;
      const float x1 = (float)((G.llam[i1 - 1] - llc) * G.inv_dllam);
      const QlgCoef cf = qlg_setup(a, qw.D, qw.SQ, S);
      const float hw = qlg_halfwidth(qw, a, S, refl, lnq);
      const int noff = (int)lroundf(fminf(fminf(hw, cap), (float)(nf + abs(ic))));
      const int fa = ic - noff > 1 ? ic - noff : 1;
      const int fb = ic + noff < nf ? ic + noff : nf;
      if (diag && lane == 0) {
        const float rch = (float)((double)hw * G.dllam);
        atomicMax(reinterpret_cast<int *>(reach + ln), __float_as_int(rch));
      }
      if (fa > fb) continue;
      if (diag && lane == 0) used[ln] = 1;
      const float x0 = x1 - (float)(i1 - fa);
      // line_scattering: an LTE line also gives (1-eps) of its profile to chi_scat
      // (bi = bj = 1 there, so chi and eta gain the profile itself)
      const bool scat = chi_scat && !nlte_line;
      for (int f = fa + lane; f <= fb; f += 32) {
        const float K = qlg_eval(tab, cf, x0 + (float)(f - fa));
        chi[f - 1] = fmaf(K, bi, chi[f - 1]);
        eta[f - 1] = fmaf(K, bj, eta[f - 1]);
        if (scat) chi_scat[f - 1] = fmaf(one_m_eps[f - 1], K, chi_scat[f - 1]);
      }
      __syncwarp();
    }
  }
}

// max |vproj| over the cells (select_lines' vmax), as the bits of a non-negative
// float: their unsigned order is the float order, so atomicMax is exact
__global__ void k_absmax(int n, const float *v, unsigned *out) {
  unsigned m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(fabsf(v[i])));
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__device__ __forceinline__ int lower_bound8(const double *a, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (a[mid] >= x) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}
__device__ __forceinline__ int upper_bound8(const double *a, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (a[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  return lo - 1;
}

// select_lines (linelist_mod.f90:1110-1142) with one warp: the slice by bisection on
// the centres with the largest reach as margin, then each line against its own
// reach; the ballot keeps the selected lines in ascending order
__global__ void k_select_lines(LineArgs L, const double *llam, int nf, const unsigned *vmax_bits, int *sel,
                               int *nsel) {
  const int lane = threadIdx.x & 31;
  float r = 0.0f;
  for (int l = lane; l < L.nline; l += 32) r = fmaxf(r, L.reach_in[l]);
  for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, o));
  const double rmax = (double)r;
  const double vmax = (double)__uint_as_float(*vmax_bits);
  const double hb1 = nf > 1 ? 0.5 * (llam[1] - llam[0]) : 0.0;
  const double hb2 = nf > 1 ? 0.5 * (llam[nf - 1] - llam[nf - 2]) : 0.0;
  const double blue = llam[0] - hb1 - vmax, red = llam[nf - 1] + hb2 + vmax;
  const int l0 = max(0, lower_bound8(L.llam0, L.nline, blue - rmax));
  const int l1 = min(L.nline - 1, upper_bound8(L.llam0, L.nline, red + rmax));
  int count = 0;
  for (int b = l0; b <= l1; b += 32) {
    const int l = b + lane;
    bool ok = l <= l1 && (L.active == nullptr || L.active[l]);
    if (ok) ok = !(L.llam0[l] + (double)L.reach_in[l] < blue || L.llam0[l] - (double)L.reach_in[l] > red);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if (ok) sel[count + __popc(m & ((1u << lane) - 1u))] = l;
    count += __popc(m);
  }
  if (lane == 0) *nsel = count;
}

__device__ __forceinline__ void stage_tables(float2 *s_tab, const float2 *tab) {
  for (int i = threadIdx.x; i < QLG_NTAB; i += blockDim.x) s_tab[i] = tab[i];
  __syncthreads();
}

// m3d_line_opacity: warp per cell, arrays in global memory
__global__ void __launch_bounds__(256) k_line_opacity(LineArgs L, GridArgs G, int ncell, float *chi, float *eta,
                                                      const float *cont, const float *logref, const float *vproj,
                                                      const float *inv_df, const float *vbar2, const float *e_kT,
                                                      const float *lnbase, const float *ne, const float *tothi,
                                                      const float *stark_pe, const float *dep_mem, int do_nlte,
                                                      int diag, uint8_t *used, float *strength, float *reach,
                                                      const float2 *tab, const float *one_m_eps, float *chi_scat) {
  extern __shared__ float smem[];
  float2 *s_tab = reinterpret_cast<float2 *>(smem);
  stage_tables(s_tab, tab);
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int cell = blockIdx.x * warps + (threadIdx.x >> 5); cell < ncell; cell += gridDim.x * warps) {
    CellArgs c;
    c.idf = inv_df[cell]; c.vbar2 = vbar2[cell]; c.ekt = e_kT[cell]; c.ne = ne[cell];
    c.tothi = tothi[cell]; c.starkpe = stark_pe[cell]; c.vproj = vproj[cell]; c.base = lnbase[cell];
    const size_t o = (size_t)G.nf * cell;
    auto dep = [&](int lev) { return dep_mem[(size_t)cell + (size_t)ncell * (size_t)(lev - 1)]; };
    warp_cell_lines(L, G, c, chi + o, eta + o, cont + o, logref + o, dep, do_nlte != 0, diag != 0, used, strength,
                    reach, s_tab, lane, one_m_eps ? one_m_eps + o : nullptr, chi_scat ? chi_scat + o : nullptr);
  }
}

// lte_background_opacities: beta, Bnu (rt_patch_mod.f90:2004-2023)
__global__ void k_lte_background(int nf, int ncell, const double *nu, const float *temp, float *beta, float *Bnu) {
  const size_t n = (size_t)nf * ncell;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(k % nf);
    const size_t i = k / nf;
    const float h_kT = (float)(M3D_H_K / (double)temp[i]);
    const float hv = (float)(nu[f] * (double)h_kT);
    float E, u0;
    exp_neg(hv, E, u0);
    const float b = fmaxf(E, FLT_MIN);
    beta[k] = b;
    Bnu[k] = b / (1.0f - b);
  }
}

// work_to_transfer_units without split rates or line scattering (rt_patch_mod.f90:3571-3651)
__global__ void k_transfer_units(size_t n, float *w1, float *w2, const float *beta, float fl, int suppress,
                                 int *n_floored) {
  int cnt = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const float xhat = w1[k];
    const float etav = w2[k] * beta[k];
    float chi = xhat - etav;
    const float floor_ = fmaxf(fl * fabsf(xhat), FLT_MIN);
    if (suppress) chi = fmaxf(chi, floor_);
    else if (fabsf(chi) < floor_) { chi = copysignf(floor_, chi); cnt++; }
    w1[k] = chi;
    w2[k] = etav / chi;
  }
  if (n_floored && cnt) atomicAdd(n_floored, cnt);
}

// integrate_intensity (rt_patch_mod.f90:3399-3431)
__global__ void k_integrate_intensity(size_t n, float wmu, const float *inu, const float *psi, float *Jnu,
                                      float *PsiJ) {
  const float w2 = 2.0f * wmu;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    Jnu[k] = fmaf(w2, inu[k], Jnu[k]);
    if (psi && PsiJ) PsiJ[k] = fmaf(w2, psi[k], PsiJ[k]);
  }
}

// ----------------------------------------------------------------------------
// Formal solvers
// ----------------------------------------------------------------------------
struct SlabArgs {
  int nf, nx, ny, nz, dir, get_psi, split_rates;
  double ds[3], vec[3];
  double maser_dtau_max, maser_Inu_max;
};

// long_char_linear (rt_solvers_mod.f90:666-757): thread per (f, x, y), z sequential
template <typename T>
__global__ void k_long_char_linear(SlabArgs s, T *work, T *psi, T *irem, T *esc, T dsup05) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nf = s.nf, nx = s.nx, ny = s.ny, nz = s.nz, dir = s.dir;
  if (g >= (size_t)nf * nx * ny) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const T dtmax = -(T)s.maser_dtau_max, Imax = (T)s.maser_Inu_max;
  const int zs = dir > 0 ? 1 : nz;
  const size_t zstride = (size_t)nf * nx * ny;
  const size_t k1 = zstride * (nz + 2);
  const size_t b = g;
  T xxup = work[b + zstride * (zs - dir)], ssup = work[b + zstride * (zs - dir) + k1];
  T Inuup = work[b + zstride * (zs - dir) + 2 * k1];
  for (int i = 0, z = zs; i < nz; i++, z += dir) {
    const size_t o = b + zstride * z;
    const T xx = work[o], ss = work[o + k1];
    T dt = dsup05 * (xxup + xx);
    dt = tmax(dt, dtmax);
    T E, W, Psi, Esc;
    linear_weights(dt, E, W, Psi, Esc);
    T Inu = fma_t(Psi, ss, fma_t(W, ssup, Inuup * E));
    if (s.split_rates) {
      const bool off = dt <= 0 || xx <= 0 || tabs(Inu) > Imax;
      const T Irem = fma_t(W, ssup, Inuup * E);
      Inu = tmax(-Imax, tmin(Imax, Inu));
      Psi = off ? (T)0 : Psi;
      const size_t p = ip(f, x, y, z, nf, nx, ny);
      irem[p] = off ? Inu : Irem;
      esc[p] = off ? (T)1 : Esc;
    } else {
      Inu = tmax(-Imax, tmin(Imax, Inu));
    }
    work[o + 2 * k1] = Inu;
    if (s.get_psi) psi[ip(f, x, y, z, nf, nx, ny)] = (dt > 0 && xx > 0) ? Psi / xx : (T)0;
    xxup = xx; ssup = ss; Inuup = Inu;
  }
}

// long_char_hermite (rt_solvers_mod.f90:1052-1504): the chain-rule cubic-Hermite
// long characteristics, one thread per (f, x, y), z sequential.  herm_dtau: dchi/ds
// at both ends by chi = (chi/Pe) Pe from a parabola through three samples,
// MC-clamped, then the Euler-Maclaurin trapezoid.  herm_source: dS/dtau by
// S = rho Bnu, the cubic-Bezier control points clamped to [min, max] of the end
// values, bezier3_weights.  herm_first: the zeroed top ghost's secant step.
// Slabs of at least 3 planes.
struct HermArgs {
  float rdsup, dsup1, dsup2, dtmax, Imax, gfac;
  int get_rates, ghost_thermo;
  const float *beta, *pe, *dpe_dz, *dlnt_dz, *temp, *hknu;
  const float *g_pe, *g_dpe_dz, *g_dlnt_dz, *g_temp;
};

__device__ __forceinline__ float herm_dtau(const HermArgs &K, float xxup, float xxc, float xx3, float peu, float rpeu,
                                           float gpu, float pec, float rpec, float gpc, float rpe3, bool center) {
  const float dtmin = 1e-20f;
  const float hh = 0.5f * K.rdsup;
  const float t1 = (xxc - xxup) * K.rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpu = xxup * rpeu, rxpc = xxc * rpec, rxp3 = xx3 * rpe3;
  float drxpu, drxpc;
  if (center) {
    drxpc = (rxp3 - rxpu) * hh;
    drxpu = (fmaf(-3.0f, rxpu, 4.0f * rxpc) - rxp3) * hh;
  } else {
    drxpu = (rxpc - rxp3) * hh;
    drxpc = fmaf(3.0f, rxpc, fmaf(-4.0f, rxpu, rxp3)) * hh;
  }
  float mup = fmaf(rxpu, gpu, peu * drxpu);
  float mc = fmaf(rxpc, gpc, pec * drxpc);
  mup = sgn * fmaxf(0.0f, fminf(sgn * mup, 2.0f * fabsf(t1)));
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 2.0f * fabsf(t1)));
  float dt = fmaf(K.dsup1, xxup + xxc, K.dsup2 * (mup - mc));
  return fmaxf(copysignf(fmaxf(fabsf(dt), dtmin), dt), K.dtmax);
}

__device__ __forceinline__ void herm_source(const HermArgs &K, float xxup, float xxc, float ssup, float ssc, float ss3,
                                            float betau, float betac, float beta3, float hk, float Inuup, float aTu,
                                            float aTc, bool center, float dt, float ex, float w0, float w1, float w2,
                                            float w3, float &Inu, float &plam) {
  const float third = 0.333333343f;
  const float hh = 0.5f * K.rdsup;
  const float r1mbu = 1.0f / (1.0f - betau), r1mbc = 1.0f / (1.0f - betac), r1mb3 = 1.0f / (1.0f - beta3);
  const float Bu = betau * r1mbu, Bc = betac * r1mbc, B3 = beta3 * r1mb3;
  const float rhou = ssup / Bu, rhoc = ssc / Bc, rho3 = ss3 / B3;
  float drhu, drhc;
  if (center) {
    drhc = (rho3 - rhou) * hh;
    drhu = (fmaf(-3.0f, rhou, 4.0f * rhoc) - rho3) * hh;
  } else {
    drhu = (rhoc - rho3) * hh;
    drhc = fmaf(3.0f, rhoc, fmaf(-4.0f, rhou, rho3)) * hh;
  }
  const float rxxu = 1.0f / xxup, rxxc = 1.0f / xxc;
  const float gu = ((hk * r1mbu) * aTu) * rxxu;
  const float gc = ((hk * r1mbc) * aTc) * rxxc;
  const float dt3 = dt * third;
  float P1 = fmaf(dt3, fmaf(ssup, gu, (Bu * drhu) * rxxu), ssup);
  float P2 = fmaf(-dt3, fmaf(ssc, gc, (Bc * drhc) * rxxc), ssc);
  const float smin = fminf(ssup, ssc), smax = fmaxf(ssup, ssc);
  P1 = fminf(fmaxf(P1, smin), smax);
  P2 = fminf(fmaxf(P2, smin), smax);
  const float I = fmaf(w3, ssc, fmaf(w2, P2, fmaf(w1, P1, fmaf(w0, ssup, Inuup * ex))));
  Inu = fmaxf(-K.Imax, fminf(K.Imax, I));
  const float d1 = fminf(fmaxf((Bu * third) / Bc, 0.0f), 1.0f);
  const float d2 = fminf(fmaxf(fmaf(-dt3, gc, 0.666666687f), 0.0f), 1.0f);
  plam = (K.get_rates && dt > 0 && xxc > 0) ? (fmaf(w1, d1, w2 * d2) + w3) * rxxc : 0.0f;
}

__device__ __forceinline__ void herm_first(const HermArgs &K, float xxup, float xxc, float xxdn, float ssup, float ssc,
                                           float ssdn, float betac, float betadn, float hk, float Inuup, float pec,
                                           float rpec, float rpedn, float gpc, float aTc, float &Inu, float &plam) {
  const float dtmin = 1e-20f, third = 0.333333343f;
  const float t1 = (xxc - xxup) * K.rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpc = xxc * rpec;
  float mc = fmaf(rxpc, gpc, (pec * fmaf(xxdn, rpedn, -rxpc)) * K.rdsup);
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 2.0f * fabsf(t1)));
  float dt = fmaf(K.dsup1, xxup + xxc, K.dsup2 * (t1 - mc));
  dt = fmaxf(copysignf(fmaxf(fabsf(dt), dtmin), dt), K.dtmax);
  float ex, w0, w1, w2, w3;
  bezier3_weights(dt, ex, w0, w1, w2, w3);
  const float r1mbc = 1.0f / (1.0f - betac), r1mbdn = 1.0f / (1.0f - betadn);
  const float Bc = betac * r1mbc, Bdn = betadn * r1mbdn;
  const float Gc = ((hk * r1mbc) * aTc) / xxc;
  const float rhoc = ssc / Bc, rhodn = ssdn / Bdn;
  float taudn = K.dsup1 * (xxc + xxdn);
  taudn = copysignf(fmaxf(fabsf(taudn), dtmin), taudn);
  const float dSc = fmaf(ssc, Gc, (Bc * (rhodn - rhoc)) / taudn);
  const float dSu = (ssc - ssup) / dt;
  const float dt3 = dt * third;
  float P1 = fmaf(dt3, dSu, ssup);
  float P2 = fmaf(-dt3, dSc, ssc);
  const float smin = fminf(ssup, ssc), smax = fmaxf(ssup, ssc);
  P1 = fminf(fmaxf(P1, smin), smax);
  P2 = fminf(fmaxf(P2, smin), smax);
  const float I = fmaf(w3, ssc, fmaf(w2, P2, fmaf(w1, P1, fmaf(w0, ssup, Inuup * ex))));
  Inu = fmaxf(-K.Imax, fminf(K.Imax, I));
  plam = (K.get_rates && dt > 0 && xxc > 0) ? (fmaf(w1, third, w2) + w3) / xxc : 0.0f;
}

__global__ void k_long_char_hermite(HermArgs K, int nf, int nx, int ny, int nz, int dir, float *work, float *psi) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= (size_t)nf * nx * ny) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const size_t plane = (size_t)nf * nx * ny, k1 = plane * (nz + 2);
  const size_t cplane = (size_t)nx * ny, cxy = (size_t)x + (size_t)nx * y;
  const int zs = dir > 0 ? 1 : nz, ze = dir > 0 ? nz : 1;
  const float hk = K.hknu[f];
  for (int i = 0, z = zs; i < nz; i++, z += dir) {
    const int zup = z - dir;
    const bool first = z == zs, last = z == ze;
    const int zt = last ? ze - 2 * dir : z + dir;
    const size_t cz = cxy + cplane * (size_t)(z - 1);
    const float pec = K.pe[cz], rpec = 1.0f / pec;
    const float gpc = K.gfac * K.dpe_dz[cz];
    const float aTc = (K.gfac * K.dlnt_dz[cz]) / K.temp[cz];
    const size_t wz = g + plane * (size_t)z, wu = g + plane * (size_t)zup;
    const size_t pz = g + plane * (size_t)(z - 1);
    float I, pl;
    if (first && !K.ghost_thermo) {
      const int zdn = z + dir;
      const size_t wd = g + plane * (size_t)zdn;
      const float rpedn = 1.0f / K.pe[cxy + cplane * (size_t)(zdn - 1)];
      herm_first(K, work[wu], work[wz], work[wd], work[wu + k1], work[wz + k1], work[wd + k1], K.beta[pz],
                 K.beta[g + plane * (size_t)(zdn - 1)], hk, work[wu + 2 * k1], pec, rpec, rpedn, gpc, aTc, I, pl);
    } else {
      float peu, rpeu, gpu, aTu, bu;
      if (first) {
        peu = K.g_pe[cxy];
        rpeu = 1.0f / peu;
        gpu = K.gfac * K.g_dpe_dz[cxy];
        const float rTup = 1.0f / K.g_temp[cxy];
        aTu = (K.gfac * K.g_dlnt_dz[cxy]) * rTup;
        bu = fmaxf(exp4(-(hk * rTup)), FLT_MIN);
      } else {
        const size_t cu = cxy + cplane * (size_t)(zup - 1);
        peu = K.pe[cu];
        rpeu = 1.0f / peu;
        gpu = K.gfac * K.dpe_dz[cu];
        aTu = (K.gfac * K.dlnt_dz[cu]) / K.temp[cu];
        bu = K.beta[g + plane * (size_t)(zup - 1)];
      }
      const float rpet = 1.0f / K.pe[cxy + cplane * (size_t)(zt - 1)];
      const size_t wt = g + plane * (size_t)zt;
      const float xxup = work[wu], xxc = work[wz];
      const float dt = herm_dtau(K, xxup, xxc, work[wt], peu, rpeu, gpu, pec, rpec, gpc, rpet, !last);
      float ex, w0, w1, w2, w3;
      bezier3_weights(dt, ex, w0, w1, w2, w3);
      herm_source(K, xxup, xxc, work[wu + k1], work[wz + k1], work[wt + k1], bu, K.beta[pz],
                  K.beta[g + plane * (size_t)(zt - 1)], hk, work[wu + 2 * k1], aTu, aTc, !last, dt, ex, w0, w1, w2,
                  w3, I, pl);
    }
    work[wz + 2 * k1] = I;
    if (psi && K.get_rates) psi[pz] = pl;
  }
}

// long_char_hermite2 (rt_solvers_mod.f90:1536-1895): the hybrid solver, one thread
// per (f, x, y), z sequential.  dtau by herm_dtau's chain rule with the control-point
// bound 3 |secant|; dtau, 1/dtau and the parabola's weights in FP64 as the reference
// declares them; the source is long_char_quadratic's parabola with dS/dtau at the
// target MC-limited from the two adjacent secants (herm2_step), on the last plane a
// one-sided difference when the third sample is a plane of the slab, and the zeroed
// top ghost's secant step (herm2_first).  ghost: 0 zeroed top, 1 neighbour, 2 bottom.
struct Herm2Args {
  float rdsup, dsup1, dsup2, Imax, gfac;
  double dtmax;
  int get_rates, ghost;
  const float *pe, *dpe_dz, *g_pe, *g_dpe_dz;
};

__device__ __forceinline__ double herm2_clamp(double dt, double dtmax) {
  return fmax(copysign(fmax(fabs(dt), (double)1e-20f), dt), dtmax);
}

__device__ __forceinline__ void herm2_weights(const Herm2Args &K, double dt, double rdt, float ex, float U0, float U1,
                                              float q, float xxc, float ssup, float ssc, float dsdtau, float Inuup,
                                              float &Inu, float &plam) {
  const double B = __dmul_rn(__dsub_rn(2.0 * (double)U1, (double)q), rdt);
  const double A = __dsub_rn((double)U0, B);
  const float C = q - U1;
  const float I = fmaf(C, dsdtau, fmaf((float)B, ssc, fmaf((float)A, ssup, Inuup * ex)));
  Inu = fmaxf(-K.Imax, fminf(K.Imax, I));
  plam = (K.get_rates && dt > 0 && xxc > 0) ? (float)B / xxc : 0.0f;
}

__device__ __forceinline__ void herm2_step(const Herm2Args &K, float xxup, float xxc, float xx3, float ssup,
                                           float ssc, float ss3, float Inuup, float peu, float rpeu, float gpu,
                                           float pec, float rpec, float gpc, float pe3, float rpe3, float gp3,
                                           bool center, bool onesided, float &Inu, float &plam) {
  const float hh = 0.5f * K.rdsup;
  const float t1 = (xxc - xxup) * K.rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpu = xxup * rpeu, rxpc = xxc * rpec, rxp3 = xx3 * rpe3;
  float drxpu, drxpc;
  if (center) {
    drxpc = (rxp3 - rxpu) * hh;
    drxpu = (fmaf(-3.0f, rxpu, 4.0f * rxpc) - rxp3) * hh;
  } else {
    drxpu = (rxpc - rxp3) * hh;
    drxpc = fmaf(3.0f, rxpc, fmaf(-4.0f, rxpu, rxp3)) * hh;
  }
  float mup = fmaf(rxpu, gpu, peu * drxpu);
  float mc = fmaf(rxpc, gpc, pec * drxpc);
  mup = sgn * fmaxf(0.0f, fminf(sgn * mup, 3.0f * fabsf(t1)));
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 3.0f * fabsf(t1)));
  const double dt = herm2_clamp((double)fmaf(K.dsup1, xxup + xxc, K.dsup2 * (mup - mc)), K.dtmax);
  const double rdt = __drcp_rn(dt);
  float ex, U0, U1, q;
  parab_moments((float)dt, ex, U0, U1, q);
  const float s1 = (ssc - ssup) * (float)rdt;
  float dsdtau = s1;
  if (center) {
    const float t3 = (xx3 - xxc) * K.rdsup;
    const float sgn3 = copysignf(1.0f, t3);
    const float drxp3 = fmaf(3.0f, rxp3, fmaf(-4.0f, rxpc, rxpu)) * hh;
    float m3 = fmaf(rxp3, gp3, pe3 * drxp3);
    m3 = sgn3 * fmaxf(0.0f, fminf(sgn3 * m3, 3.0f * fabsf(t3)));
    const double dt3 = herm2_clamp((double)fmaf(K.dsup1, xxc + xx3, K.dsup2 * (mc - m3)), K.dtmax);
    const float s3 = (ss3 - ssc) / (float)dt3;
    const float avg = 0.5f * (s1 + s3);
    dsdtau = (copysignf(1.0f, s1) + copysignf(1.0f, s3)) * fminf(fminf(fabsf(s1), fabsf(s3)), fabsf(0.5f * avg));
  } else if (onesided && xxc > 0.0f) {
    const float d = (fmaf(3.0f, ssc, fmaf(-4.0f, ssup, ss3)) * hh) / xxc;
    const float sg = copysignf(1.0f, s1);
    dsdtau = sg * fmaxf(0.0f, fminf(sg * d, 2.0f * fabsf(s1)));
  }
  herm2_weights(K, dt, rdt, ex, U0, U1, q, xxc, ssup, ssc, dsdtau, Inuup, Inu, plam);
}

__device__ __forceinline__ void herm2_first(const Herm2Args &K, float xxup, float xxc, float xxdn, float ssup,
                                            float ssc, float Inuup, float pec, float rpec, float rpedn, float gpc,
                                            float &Inu, float &plam) {
  const float t1 = (xxc - xxup) * K.rdsup;
  const float sgn = copysignf(1.0f, t1);
  const float rxpc = xxc * rpec;
  float mc = fmaf(rxpc, gpc, (pec * fmaf(xxdn, rpedn, -rxpc)) * K.rdsup);
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 3.0f * fabsf(t1)));
  const double dt = herm2_clamp((double)fmaf(K.dsup1, xxup + xxc, K.dsup2 * (t1 - mc)), K.dtmax);
  const double rdt = __drcp_rn(dt);
  float ex, U0, U1, q;
  parab_moments((float)dt, ex, U0, U1, q);
  const float dsdtau = (ssc - ssup) * (float)rdt;
  herm2_weights(K, dt, rdt, ex, U0, U1, q, xxc, ssup, ssc, dsdtau, Inuup, Inu, plam);
}

__global__ void k_long_char_hermite2(Herm2Args K, int nf, int nx, int ny, int nz, int dir, float *work, float *psi) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= (size_t)nf * nx * ny) return;
  const int x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const size_t plane = (size_t)nf * nx * ny, k1 = plane * (nz + 2);
  const size_t cplane = (size_t)nx * ny, cxy = (size_t)x + (size_t)nx * y;
  const int zs = dir > 0 ? 1 : nz, ze = dir > 0 ? nz : 1;
  for (int i = 0, z = zs; i < nz; i++, z += dir) {
    const int zup = z - dir;
    const bool first = z == zs, last = z == ze;
    const size_t cz = cxy + cplane * (size_t)(z - 1);
    const float pec = K.pe[cz], rpec = 1.0f / pec;
    const float gpc = K.gfac * K.dpe_dz[cz];
    float peu = 0.0f, rpeu = 0.0f, gpu = 0.0f;
    if (first && K.ghost) {
      peu = K.g_pe[cxy];
      rpeu = 1.0f / peu;
      gpu = K.gfac * K.g_dpe_dz[cxy];
    } else if (!first) {
      const size_t cu = cxy + cplane * (size_t)(zup - 1);
      peu = K.pe[cu];
      rpeu = 1.0f / peu;
      gpu = K.gfac * K.dpe_dz[cu];
    }
    const int z3 = last ? z - 2 * dir : z + dir;
    float pe3 = 0.0f, rpe3, gp3 = 0.0f;
    if (!last) {
      const size_t c3 = cxy + cplane * (size_t)(z3 - 1);
      pe3 = K.pe[c3];
      rpe3 = 1.0f / pe3;
      gp3 = K.gfac * K.dpe_dz[c3];
    } else if (nz >= 3) {
      rpe3 = 1.0f / K.pe[cxy + cplane * (size_t)(z3 - 1)];
    } else {
      rpe3 = K.ghost == 1 ? 1.0f / K.g_pe[cxy] : rpec;
    }
    const size_t wz = g + plane * (size_t)z, wu = g + plane * (size_t)zup, w3 = g + plane * (size_t)z3;
    float I, pl;
    if (first && !K.ghost)
      herm2_first(K, work[wu], work[wz], work[w3], work[wu + k1], work[wz + k1], work[wu + 2 * k1], pec, rpec, rpe3,
                  gpc, I, pl);
    else
      herm2_step(K, work[wu], work[wz], work[w3], work[wu + k1], work[wz + k1], work[w3 + k1], work[wu + 2 * k1], peu,
                 rpeu, gpu, pec, rpec, gpc, pe3, rpe3, gp3, !last, last && nz >= 3, I, pl);
    work[wz + 2 * k1] = I;
    if (psi && K.get_rates) psi[g + plane * (size_t)(z - 1)] = pl;
  }
}

template <typename T>
__device__ __forceinline__ T dt500_of(double dsup, double c, double cu) {
  const double r = cu / c;
  if (fabs(r - 1.0) < 1e-3) return (T)(dsup * c * (1.0 + (r - 1.0) * (0.5 - (r - 1.0) / 12.0)));
  return (T)(dsup * c * (r - 1.0) / log(r));
}

// The update of one point shared by long_char2 and short_char2 once the upwind
// values are known (rt_solvers_mod.f90:404-491 and :606-657).
template <typename T>
__device__ __forceinline__ void linear2_point(bool split, int row, bool special, T xxup, T eup, T Inuup, T ssup,
                                              T chi, T ss, T xx, T dt, T d5, T rc, T Imax, T &Inu_out,
                                              T &psi_out, T &irem_out, T &esc_out) {
  T E, W, Psi, Esc;
  linear_weights(dt, E, W, Psi, Esc);
  const T pl = Psi / tcopysign(tmax(tabs(chi), tiny_of<T>()), chi);
  if (split && row == 0) {
    const T Irem = fma_t(W, ssup, Inuup * E);
    T Inu = fma_t(Psi, ss, Irem);
    const bool off = tmin(tmin(dt, chi), Imax - tabs(Inu)) <= 0;
    Inu = tmax(-Imax, tmin(Imax, Inu));
    irem_out = off ? Inu : Irem;
    esc_out = off ? (T)1 : Esc;
    Inu_out = Inu;
    psi_out = off ? (T)0 : pl;
  } else if (split) {
    const T ee = xx * ss;
    const T rxb = d5 / (dt != 0 ? dt : (T)1);
    const T Irem = special ? fma_t(W * eup, rxb, Inuup * E) : fma_t(W, ssup, Inuup * E);
    T Inu = special ? fma_t(Psi * ee, rxb, Irem) : fma_t(Psi, ss, Irem);
    T mm = tmin(tmin(dt, chi), Imax - tabs(Inu));
    mm = tmin(mm, special ? xxup : (T)1);
    const bool off = mm <= 0;
    Esc = special ? fma_t(((T)0.5 * Psi) * (xxup - xx), rxb, Esc) : Esc;
    Inu = tmax(-Imax, tmin(Imax, Inu));
    irem_out = off ? Inu : Irem;
    esc_out = off ? (T)1 : Esc;
    Inu_out = Inu;
    psi_out = off ? (T)0 : (special ? (Psi * rxb) * rc : pl);
  } else if (row == 0) {
    const T Inu = fma_t(Psi, ss, fma_t(W, ssup, Inuup * E));
    Inu_out = tmax(-Imax, tmin(Imax, Inu));
    const bool off = tmin(dt, chi) <= 0;
    psi_out = off ? (T)0 : pl;
  } else {
    const T ee = xx * ss;
    const T rxb = d5 / (dt != 0 ? dt : (T)1);
    const T Inu = special ? fma_t(fma_t(Psi, ee, W * eup), rxb, Inuup * E) : fma_t(Psi, ss, fma_t(W, ssup, Inuup * E));
    Inu_out = tmax(-Imax, tmin(Imax, Inu));
    T mm = tmin(dt, chi);
    mm = tmin(mm, special ? xxup : (T)1);
    const bool off = mm <= 0;
    psi_out = off ? (T)0 : (special ? (Psi * rxb) * rc : pl);
  }
}

// long_char2 (rt_solvers_mod.f90:527-663)
template <typename T>
__global__ void k_long_char2(SlabArgs s, T *work, T *psi, T *irem, T *esc, const float *chi500, const float *g500,
                             const int *eta_row, const uint8_t *eta_mask, double dsup) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nf = s.nf, nx = s.nx, ny = s.ny, nz = s.nz, dir = s.dir;
  if (g >= (size_t)nf * nx * ny) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const T dtmax = -(T)s.maser_dtau_max, Imax = (T)s.maser_Inu_max;
  const int zs = dir > 0 ? 1 : nz;
  const size_t zstride = (size_t)nf * nx * ny;
  const size_t k1 = zstride * (nz + 2);
  for (int i = 0, z = zs; i < nz; i++, z += dir) {
    const int zup = z - dir;
    const double c = chi500[ic3(x, y, z, nx, ny)];
    const double cu = (zup < 1 || zup > nz) ? (double)g500[x + nx * y] : (double)chi500[ic3(x, y, zup, nx, ny)];
    const T d5 = dt500_of<T>(dsup, c, cu);
    const T rc = (T)(1.0 / c), rcu = (T)(1.0 / cu);
    const int row = eta_row ? eta_row[ic3(x, y, z, nx, ny)] : 0;
    const bool special = row > 0 ? eta_mask[(size_t)f + (size_t)nf * (size_t)(row - 1)] != 0 : false;
    const size_t ou = g + zstride * zup, o = g + zstride * z;
    const T xxup = work[ou] * rcu, ssup = work[ou + k1], Inuup = work[ou + 2 * k1];
    const T eup = xxup * ssup;
    const T chi = work[o], ss = work[o + k1];
    const T xx = chi * rc;
    const T dt = tmax(((T)0.5 * (xxup + xx)) * d5, dtmax);
    T Inu, ps, ir = 0, es = 0;
    linear2_point<T>(s.split_rates != 0, row, special, xxup, eup, Inuup, ssup, chi, ss, xx, dt, d5, rc, Imax, Inu,
                     ps, ir, es);
    work[o + 2 * k1] = Inu;
    const size_t p = ip(f, x, y, z, nf, nx, ny);
    if (s.split_rates) { irem[p] = ir; esc[p] = es; }
    if (s.get_psi) psi[p] = ps;
  }
}

// quad_step of long_char_quadratic (rt_solvers_mod.f90:966-1019)
// the step from the two slopes of the extinction on, t1 = (xxc - xxup) rdsup and
// t3 = (xxdn - xxc) rdsup (a sweep carries t3 into the next step's t1: same operands)
template <typename T>
__device__ __forceinline__ void quad_step_t13(T t1, T t3, T xxup, T xxc, T xxdn, T ssup, T ssc, T ssdn, T Inuup,
                                              bool at_target, T dsup1, T dsup2, T dtmax, T Imax, bool get_psi,
                                              T &Inu_out, T &plam_out) {
  const T dtmin = (T)1e-20f;
  T t2 = (T)0.5 * (t1 + t3);
  t2 = (tcopysign((T)1, t1) + tcopysign((T)1, t3)) * tmin(tmin(tabs(t1), tabs(t3)), tabs((T)0.5 * t2));
  T dtup = fma_t(dsup2, t1 - t2, dsup1 * (xxup + xxc));
  T dtdn = fma_t(dsup2, t2 - t3, dsup1 * (xxdn + xxc));
  dtup = tmax(tcopysign(tmax(tabs(dtup), dtmin), dtup), dtmax);
  dtdn = tmax(tcopysign(tmax(tabs(dtdn), dtmin), dtdn), dtmax);
  const T dt = at_target ? dtup : dtdn;
  const T rdt = recip(dt);
  T ex, U0, U1, q;
  parab_moments(dt, ex, U0, U1, q);
  if (at_target) {
    t1 = (ssc - ssup) * rdt;
    t3 = (ssdn - ssc) / dtdn;
  } else {
    t1 = (ssc - ssup) / dtup;
    t3 = (ssdn - ssc) * rdt;
  }
  t2 = (T)0.5 * (t1 + t3);
  const T dsdtau = (tcopysign((T)1, t1) + tcopysign((T)1, t3)) * tmin(tmin(tabs(t1), tabs(t3)), tabs((T)0.5 * t2));
  T plam = 0, Inu;
  if (at_target) {
    const T B = ((T)2 * U1 - q) * rdt;
    const T A = U0 - B;
    const T C = q - U1;
    Inu = fma_t(C, dsdtau, fma_t(B, ssc, fma_t(A, ssup, Inuup * ex)));
    if (get_psi && dt > 0 && xxc > 0) plam = B / xxc;
  } else {
    const T A = q * rdt;
    const T B = U0 - A;
    const T C = U1 - q;
    Inu = fma_t(C, dsdtau, fma_t(B, ssc, fma_t(A, ssdn, Inuup * ex)));
    if (get_psi && dt > 0 && xxdn > 0) plam = A / xxdn;
  }
  Inu_out = tmax(-Imax, tmin(Imax, Inu));
  plam_out = plam;
}

template <typename T>
__device__ __forceinline__ void quad_step(T xxup, T xxc, T xxdn, T ssup, T ssc, T ssdn, T Inuup, bool at_target,
                                          T rdsup, T dsup1, T dsup2, T dtmax, T Imax, bool get_psi, T &Inu_out,
                                          T &plam_out) {
  const T t1 = (xxc - xxup) * rdsup;
  const T t3 = (xxdn - xxc) * rdsup;
  quad_step_t13<T>(t1, t3, xxup, xxc, xxdn, ssup, ssc, ssdn, Inuup, at_target, dsup1, dsup2, dtmax, Imax, get_psi,
                   Inu_out, plam_out);
}

struct QuadConst { float rdsup, dsup1, dsup2; };

// long_char_quadratic (rt_solvers_mod.f90:891-1020) on a slab's work array
template <typename T>
__global__ void k_long_char_quadratic(SlabArgs s, T *work, T *psi, QuadConst qc) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nf = s.nf, nx = s.nx, ny = s.ny, nz = s.nz, dir = s.dir;
  if (g >= (size_t)nf * nx * ny) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const T dtmax = -(T)s.maser_dtau_max, Imax = (T)s.maser_Inu_max;
  const T rdsup = (T)qc.rdsup, dsup1 = (T)qc.dsup1, dsup2 = (T)qc.dsup2;
  const bool gp = s.get_psi != 0;
  const int zs = dir > 0 ? 1 : nz, ze = dir > 0 ? nz : 1;
  const size_t zstride = (size_t)nf * nx * ny;
  const size_t k1 = zstride * (nz + 2);
  T xu = work[g + zstride * (zs - dir)], su = work[g + zstride * (zs - dir) + k1];
  T Iu = work[g + zstride * (zs - dir) + 2 * k1];
  T xc = work[g + zstride * zs], sc = work[g + zstride * zs + k1];
  T xd = work[g + zstride * (zs + dir)], sd = work[g + zstride * (zs + dir) + k1];
  int z = zs;
  for (; z != ze; z += dir) {
    T Inu, pl;
    quad_step<T>(xu, xc, xd, su, sc, sd, Iu, true, rdsup, dsup1, dsup2, dtmax, Imax, gp, Inu, pl);
    work[g + zstride * z + 2 * k1] = Inu;
    if (gp) psi[ip(f, x, y, z, nf, nx, ny)] = pl;
    Iu = Inu;
    if (z + dir != ze) {
      xu = xc; su = sc; xc = xd; sc = sd;
      xd = work[g + zstride * (z + 2 * dir)];
      sd = work[g + zstride * (z + 2 * dir) + k1];
    }
  }
  // last plane: the interval z0 -> ze with dS/dtau at its upwind end z0; the
  // planes (ze-2dir, ze-dir, ze) are the ones held after the final interior step
  {
    T Inu, pl;
    quad_step<T>(xu, xc, xd, su, sc, sd, Iu, false, rdsup, dsup1, dsup2, dtmax, Imax, gp, Inu, pl);
    work[g + zstride * ze + 2 * k1] = Inu;
    if (gp) psi[ip(f, x, y, ze, nf, nx, ny)] = pl;
  }
}

// rotate_array (rt_patch_mod.f90:3809-3866) of plane z of slot k, out of place
struct RotPlane { int up1, up2; float a, b, c, d; };

template <typename T>
__global__ void k_rotate_planes(int nf, int nx, int ny, int nz, const T *src, T *dst, const RotPlane *rot) {
  // src, dst: (nf, nx, ny, nz) views of planes 1..nz of one slot of work
  const size_t plane = (size_t)nf * nx * ny;
  const size_t n = plane * nz;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
    const size_t inplane = g % plane;
    const int z = (int)(g / plane);
    const int f = (int)(inplane % nf), x = (int)((inplane / nf) % nx), y = (int)(inplane / ((size_t)nf * nx));
    const RotPlane r = rot[z];
    const int x1 = wrap(x + r.up1, nx), x2 = wrap(x + r.up1 + 1, nx);
    const int y1 = wrap(y + r.up2, ny), y2 = wrap(y + r.up2 + 1, ny);
    const T *p = src + plane * (size_t)z;
    T v = (T)r.a * p[(size_t)f + (size_t)nf * ((size_t)x1 + (size_t)nx * y1)];
    v = fma_t((T)r.b, p[(size_t)f + (size_t)nf * ((size_t)x2 + (size_t)nx * y1)], v);
    v = fma_t((T)r.c, p[(size_t)f + (size_t)nf * ((size_t)x1 + (size_t)nx * y2)], v);
    v = fma_t((T)r.d, p[(size_t)f + (size_t)nf * ((size_t)x2 + (size_t)nx * y2)], v);
    dst[g] = v;
  }
}

// set_upstream_boundary (rt_patch_mod.f90:3270-3393) on the ghost plane of work
struct PchipConst { float c0, p, cm0, cm1, dx1; };

template <typename T>
__global__ void k_upstream_boundary(int nf, int nx, int ny, int nz, int dir, T *work, int mode, const T *mem,
                                    PchipConst pc, const float *ghost_r500, const float *ghost_temp,
                                    const double *nu) {
  const size_t plane = (size_t)nf * nx * ny;
  const int z = dir > 0 ? 0 : nz + 1, zi = dir > 0 ? 1 : -1;
  const size_t k1 = plane * (nz + 2);
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < plane; g += (size_t)gridDim.x * blockDim.x) {
  const size_t o = g + plane * z;
  if (mode == 1) {
    work[o] = 0; work[o + k1] = 0; work[o + 2 * k1] = 0;
  } else if (mode == 2) {
    for (int k = 0; k < 2; k++) {
      const float y1 = (float)work[g + plane * (z + zi) + k * k1], y2 = (float)work[g + plane * (z + 2 * zi) + k * k1];
      const float dy1 = y2 - y1;
      const float dydx1 = (2.0f * dy1) / pc.dx1 - 0.0f;
      const float v = (pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * dydx1 + pc.cm1 * 0.0f);
      work[o + k * k1] = (T)fmaxf(v, 0.0f);
    }
    work[o + 2 * k1] = work[o + k1];
  } else if (mode == 3) {
    const int f = (int)(g % nf);
    const size_t xy = g / nf;
    const float r500 = ghost_r500[xy];
    const float h_kT = (float)(M3D_H_K / (double)ghost_temp[xy]);
    const float hv = (float)(nu[f] * (double)h_kT);
    float E, u0;
    exp_neg(hv, E, u0);
    const float beta = fmaxf(E, FLT_MIN);
    work[o] = work[g + plane * (z + zi)] * (T)r500;
    work[o + k1] = (T)(beta / (1.0f - beta));
    work[o + 2 * k1] = work[o + k1];
  } else {
    work[o] = mem[g]; work[o + k1] = mem[g + plane]; work[o + 2 * k1] = mem[g + 2 * plane];
  }
  }
}


// short_char (rt_solvers_mod.f90:19-189) on one plane z: the 4x4 cubic upwind
// interpolation of chi, S and I (the row pass, then the column pass), clamped
// below by the inner 2x2 minimum; dt = dsup/2 (chi_up + chi) capped at
// -maser_dtau_max; the linear step, I clamped to +-maser_Inu_max; Psi/chi, and Irem
// and the escape factor for split rates.  Tiled: a block takes SC_TX x SC_TY
// columns of SC_TF frequencies and stages the upstream (SC_TX+3) x (SC_TY+3)
// patch of chi, S and I in shared memory once (every upstream value feeds up to
// 16 stencils).  The upwind
// tables are xt[4x+ii] = (xt[0] + x + ii) mod nx, so a tile's stencils cover
// consecutive upstream columns starting at xt[4 x0].
constexpr int SC_TX = 8, SC_TY = 8, SC_TF = 32;

// one element global -> shared without a register round trip (cp.async, sm_80+);
// all of a block's copies are in flight together and complete at cp_async_wait_all
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(sizeof(T)));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <typename T>
__global__ void __launch_bounds__(256) k_short_char_tile(SlabArgs s, int z, T *work, T *psi, T *irem, T *esc,
                                                         const int *xt, const int *yt, float4 kx, float4 ky,
                                                         T dsup05) {
  extern __shared__ __align__(16) unsigned char sc_smem[];
  T *up = (T *)sc_smem;  // [3][SC_TY+3][SC_TX+3][SC_TF]
  constexpr int PX = SC_TX + 3, PY = SC_TY + 3;
  __shared__ int sxu[PX], syu[PY];
  const int nf = s.nf, nx = s.nx, ny = s.ny, nz = s.nz, dir = s.dir;
  const int ntx = (nx + SC_TX - 1) / SC_TX, nty = (ny + SC_TY - 1) / SC_TY;
  const int bt = blockIdx.x;
  const int tx = bt % ntx, ty = (bt / ntx) % nty, fc = bt / (ntx * nty);
  const int x0 = tx * SC_TX, y0 = ty * SC_TY, f0 = fc * SC_TF;
  const int zup = z - dir;
  if (threadIdx.x < PX) sxu[threadIdx.x] = (xt[4 * x0] + threadIdx.x) % nx;
  else if (threadIdx.x < PX + PY) syu[threadIdx.x - PX] = (yt[4 * y0] + threadIdx.x - PX) % ny;
  __syncthreads();
  // one warp per upstream row of SC_TF frequencies (coalesced)
  {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool fin = f0 + lane < nf && lane < SC_TF;
    const size_t plane = (size_t)nf * nx * ny, slot = plane * (nz + 2);
    for (int row = wid; row < 3 * PY * PX; row += nw) {
      const int xi = row % PX, yj = (row / PX) % PY, i = row / (PX * PY);
      const size_t base = slot * i + plane * zup + (size_t)nf * (sxu[xi] + (size_t)nx * syu[yj]) + f0;
      if (fin) cp_async_elem(&up[row * SC_TF + lane], &work[base + lane]);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  const T dtmax = -(T)s.maser_dtau_max, Imax = (T)s.maser_Inu_max;
  const T k_x[4] = {(T)kx.x, (T)kx.y, (T)kx.z, (T)kx.w};
  const T k_y[4] = {(T)ky.x, (T)ky.y, (T)ky.z, (T)ky.w};
  // one warp per column x of the tile, lanes along f, sliding down y: the row sums
  // of an upstream row serve the four targets whose stencils hold it
  const int lane = threadIdx.x & 31, xl = threadIdx.x >> 5;
  const int x = x0 + xl, f = lane;
  if (x >= nx || f0 + f >= nf || xl >= SC_TX) return;
  const size_t plane = (size_t)nf * nx * ny, k1 = plane * (nz + 2);
  const size_t pz = plane * (size_t)z, pp = plane * (size_t)(z - 1);
  constexpr int RS = PX * SC_TF;   // one upstream row in shared memory
  constexpr int FS = PY * RS;      // one field
  const T *u0 = up + (size_t)xl * SC_TF + f;
  // window of the four upstream rows yl..yl+3: row sums, and the two inner values
  T rr[3][4], v1[3][4], v2[3][4];
  auto load_row = [&](int r, int slot) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const T *row = u0 + (size_t)i * FS + (size_t)r * RS;
      T a = 0;
#pragma unroll
      for (int ii = 0; ii < 4; ii++) a = fma_t(k_x[ii], row[ii * SC_TF], a);
      rr[i][slot] = a;
      v1[i][slot] = row[1 * SC_TF];
      v2[i][slot] = row[2 * SC_TF];
    }
  };
  // this column's chi and S on plane z for all the tile's rows, loaded up front
  T xxv[SC_TY], ssv[SC_TY];
#pragma unroll
  for (int yl = 0; yl < SC_TY; yl++) {
    const int y = y0 + yl < ny ? y0 + yl : ny - 1;
    const size_t o = pz + (size_t)nf * ((size_t)x + (size_t)nx * (size_t)y) + (size_t)(f0 + f);
    xxv[yl] = work[o];
    ssv[yl] = work[o + k1];
  }
#pragma unroll
  for (int jj = 0; jj < 3; jj++) load_row(jj, jj);
#pragma unroll
  for (int yl = 0; yl < SC_TY; yl++) {
    const int y = y0 + yl;
    if (y >= ny) break;
    load_row(yl + 3, 3);
    T upv[3], mn[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      T r = 0;
#pragma unroll
      for (int jj = 0; jj < 4; jj++) r = fma_t(k_y[jj], rr[i][jj], r);
      T m = (T)FLT_MAX;
      if (sizeof(T) == 8) m = (T)DBL_MAX;
      m = tmin(m, v1[i][1]);
      m = tmin(m, v2[i][1]);
      m = tmin(m, v1[i][2]);
      m = tmin(m, v2[i][2]);
      upv[i] = r;
      mn[i] = m;
    }
    const T xxup = tmax(upv[0], mn[0]), ssup = tmax(upv[1], mn[1]), Inuup = tmax(upv[2], mn[2]);
    const size_t col = (size_t)nf * ((size_t)x + (size_t)nx * (size_t)y) + (size_t)(f0 + f);
    const size_t o = pz + col;
    const T xx = xxv[yl], ss = ssv[yl];
    T dt = dsup05 * (xxup + xx);
    dt = tmax(dt, dtmax);
    T E, W, Psi, Esc;
    linear_weights(dt, E, W, Psi, Esc);
    T Inu = fma_t(Psi, ss, fma_t(W, ssup, Inuup * E));
    const size_t p = pp + col;
    if (s.split_rates) {
      const bool off = dt <= 0 || xx <= 0 || tabs(Inu) > Imax;
      const T Irem = fma_t(W, ssup, Inuup * E);
      Inu = tmax(-Imax, tmin(Imax, Inu));
      Psi = off ? (T)0 : Psi;
      irem[p] = off ? Inu : Irem;
      esc[p] = off ? (T)1 : Esc;
    } else {
      Inu = tmax(-Imax, tmin(Imax, Inu));
    }
    work[o + 2 * k1] = Inu;
    if (s.get_psi) psi[p] = (dt > 0 && xx > 0) ? Psi / xx : (T)0;
    // slide the window down one row
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int jj = 0; jj < 3; jj++) {
        rr[i][jj] = rr[i][jj + 1];
        v1[i][jj] = v1[i][jj + 1];
        v2[i][jj] = v2[i][jj + 1];
      }
  }
}

// short_char2 (rt_solvers_mod.f90:224-507) on plane z: each thread forms the row
// sums of its four upwind rows itself, in the reference's order (row pass, then
// column pass)
template <typename T>
__global__ void k_short_char2_plane(SlabArgs s, int z, T *work, T *psi, T *irem, T *esc, const int *xt, const int *yt,
                                    float4 kx, float4 ky, float hx, float hy, const float *chi500,
                                    const float *chi500_up, const float *g500, const int *eta_row,
                                    const uint8_t *eta_mask, double dsup) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nf = s.nf, nx = s.nx, ny = s.ny, nz = s.nz, dir = s.dir;
  if (g >= (size_t)nf * nx * ny) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const int zup = z - dir;
  const T dtmax = -(T)s.maser_dtau_max, Imax = (T)s.maser_Inu_max;
  const size_t k1 = (size_t)nf * nx * ny * (nz + 2);
  const bool ghost = zup < 1 || zup > nz;
  const int x1 = xt[4 * x], x2 = xt[4 * x + 1], x3 = xt[4 * x + 2], x4 = xt[4 * x + 3];
  const int yy[4] = {yt[4 * y], yt[4 * y + 1], yt[4 * y + 2], yt[4 * y + 3]};
  const T hxr = (T)hx, hx1 = (T)(1.0f - hx), hyr = (T)hy, hy1 = (T)(1.0f - hy);
  // row sums at the four upwind rows (row_red slots 1..4, rt_solvers_mod.f90:334-348)
  T r0[4], r1[4], r2[4], r3[4];
  for (int jj = 0; jj < 4; jj++) {
    const int yu = yy[jj];
    const float c2 = ghost ? g500[x2 + nx * yu] : chi500[ic3(x2, yu, zup, nx, ny)];
    const float c3 = ghost ? g500[x3 + nx * yu] : chi500[ic3(x3, yu, zup, nx, ny)];
    const T w2 = (T)((1.0f - hx) * (1.0f / c2));
    const T w3 = (T)(hx * (1.0f / c3));
    const T a21 = work[iw(f, x2, yu, zup, 0, nf, nx, ny, nz)], a31 = work[iw(f, x3, yu, zup, 0, nf, nx, ny, nz)];
    const T a22 = work[iw(f, x2, yu, zup, 1, nf, nx, ny, nz)], a32 = work[iw(f, x3, yu, zup, 1, nf, nx, ny, nz)];
    r0[jj] = fma_t(w3, a31, w2 * a21);
    r1[jj] = fma_t(w3 * a31, a32, (w2 * a21) * a22);
    T t = (T)kx.x * work[iw(f, x1, yu, zup, 2, nf, nx, ny, nz)];
    t = fma_t((T)kx.y, work[iw(f, x2, yu, zup, 2, nf, nx, ny, nz)], t);
    t = fma_t((T)kx.z, work[iw(f, x3, yu, zup, 2, nf, nx, ny, nz)], t);
    t = fma_t((T)kx.w, work[iw(f, x4, yu, zup, 2, nf, nx, ny, nz)], t);
    r2[jj] = t;
    r3[jj] = fma_t(hxr, a32, hx1 * a22);
  }
  const double c = chi500[ic3(x, y, z, nx, ny)];
  const double cu = chi500_up[ic3(x, y, z, nx, ny)];
  const T d5 = dt500_of<T>(dsup, c, cu);
  const T rc = (T)(1.0 / c);
  const T xxup = fma_t(hyr, r0[2], hy1 * r0[1]);
  const T eup = fma_t(hyr, r1[2], hy1 * r1[1]);
  T Inuup = (T)ky.x * r2[0];
  Inuup = fma_t((T)ky.y, r2[1], Inuup);
  Inuup = fma_t((T)ky.z, r2[2], Inuup);
  Inuup = fma_t((T)ky.w, r2[3], Inuup);
  const T m = tmin(tmin(tmin(work[iw(f, x2, yy[1], zup, 2, nf, nx, ny, nz)], work[iw(f, x3, yy[1], zup, 2, nf, nx, ny, nz)]),
                        work[iw(f, x2, yy[2], zup, 2, nf, nx, ny, nz)]),
                   work[iw(f, x3, yy[2], zup, 2, nf, nx, ny, nz)]);
  Inuup = tmax(Inuup, m);
  const size_t o = iw(f, x, y, z, 0, nf, nx, ny, nz);
  const T chi = work[o], ss = work[o + k1];
  const T xx = chi * rc;
  const T dt = tmax(((T)0.5 * (xxup + xx)) * d5, dtmax);
  const T ssup = fma_t(hyr, r3[2], hy1 * r3[1]);
  const int row = eta_row ? eta_row[ic3(x, y, z, nx, ny)] : 0;
  const bool special = row > 0 ? eta_mask[(size_t)f + (size_t)nf * (size_t)(row - 1)] != 0 : false;
  T Inu, ps, ir = 0, es = 0;
  linear2_point<T>(s.split_rates != 0, row, special, xxup, eup, Inuup, ssup, chi, ss, xx, dt, d5, rc, Imax, Inu, ps,
                   ir, es);
  work[o + 2 * k1] = Inu;
  const size_t p = ip(f, x, y, z, nf, nx, ny);
  if (s.split_rates) { irem[p] = ir; esc[p] = es; }
  if (s.get_psi) psi[p] = ps;
}

// short_char_hermite (rt_solvers_mod.f90:1917-2248) for plane z: one thread per
// (f, x, y).  short_char's 4x4 kernel sums and 2x2 minimum, past the first plane
// also over the ratios chi/Pe and Snu/Bnu formed at the upwind nodes, in the same
// order as the row pass and the column pass (a fused multiply-add per tap from
// zero); then the quadratic weights with the product-rule slopes at the target,
// dtau and the weights in FP64 as declared there, the positivity clamp of dS/dtau
// resolved by branch so the Lambda diagonal B + C kf follows it.  The first plane
// takes short_char's linear step.
struct SCHermArgs {
  float4 kx, ky;
  float v1, v2, v3, dsup05, rpath, dsc2, dtmaxf, Imax;
  double dtmax;
  const int *xt, *yt;
  const float *beta, *pe, *dpe_dx, *dpe_dy, *dpe_dz, *dlnt_dx, *dlnt_dy, *dlnt_dz, *temp, *hknu;
};

__global__ void __launch_bounds__(256) k_short_char_hermite_plane(SlabArgs s, SCHermArgs K, int z, float *work,
                                                                  float *psi, float *irem, float *esc) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int nf = s.nf, nx = s.nx, ny = s.ny, nz = s.nz, dir = s.dir;
  if (g >= (size_t)nf * nx * ny) return;
  const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
  const int zup = z - dir;
  const bool chain = z != (dir > 0 ? 1 : nz);
  const float kx[4] = {K.kx.x, K.kx.y, K.kx.z, K.kx.w}, ky[4] = {K.ky.x, K.ky.y, K.ky.z, K.ky.w};
  const size_t k1 = (size_t)nf * nx * ny * (nz + 2);
  float up[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float mn[5] = {FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX};
  const int nfld = chain ? 5 : 3;
  for (int jj = 0; jj < 4; jj++) {
    const int yu = K.yt[4 * y + jj];
    float row[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (int ii = 0; ii < 4; ii++) {
      const int xu = K.xt[4 * x + ii];
      const size_t o = iw(f, xu, yu, zup, 0, nf, nx, ny, nz);
      float v[5];
      v[0] = work[o];
      v[1] = work[o + k1];
      v[2] = work[o + 2 * k1];
      v[3] = v[4] = 0.0f;
      if (chain) {
        const float rpe = 1.0f / K.pe[ic3(xu, yu, zup, nx, ny)];
        const float bet = K.beta[ip(f, xu, yu, zup, nf, nx, ny)];
        v[3] = v[0] * rpe;
        v[4] = (v[1] * (1.0f - bet)) / bet;
      }
      const bool inner = jj >= 1 && jj <= 2 && ii >= 1 && ii <= 2;
#pragma unroll
      for (int i = 0; i < 5; i++) {
        if (i >= nfld) break;
        row[i] = fmaf(kx[ii], v[i], row[i]);
        if (inner) mn[i] = fminf(mn[i], v[i]);
      }
    }
#pragma unroll
    for (int i = 0; i < 5; i++)
      if (i < nfld) up[i] = fmaf(ky[jj], row[i], up[i]);
  }
#pragma unroll
  for (int i = 0; i < 5; i++)
    if (i < nfld) up[i] = fmaxf(up[i], mn[i]);
  const float xxup = up[0], ssup = up[1], Inuup = up[2];
  const size_t o = iw(f, x, y, z, 0, nf, nx, ny, nz);
  const float xx = work[o], ss = work[o + k1];
  const size_t p = ip(f, x, y, z, nf, nx, ny);
  const float Imax = K.Imax;
  if (!chain) {
    const float dt = fmaxf(K.dsup05 * (xxup + xx), K.dtmaxf);
    float E, W, Psi, Esc;
    linear_weights(dt, E, W, Psi, Esc);
    float Inu = fmaf(Psi, ss, fmaf(W, ssup, Inuup * E));
    if (s.split_rates) {
      const bool off = dt <= 0 || xx <= 0 || fabsf(Inu) > Imax;
      const float Irem = fmaf(W, ssup, Inuup * E);
      Inu = fmaxf(-Imax, fminf(Imax, Inu));
      Psi = off ? 0.0f : Psi;
      irem[p] = off ? Inu : Irem;
      esc[p] = off ? 1.0f : Esc;
    } else {
      Inu = fmaxf(-Imax, fminf(Imax, Inu));
    }
    work[o + 2 * k1] = Inu;
    if (s.get_psi) psi[p] = (dt > 0 && xx > 0) ? Psi / xx : 0.0f;
    return;
  }
  const size_t c = ic3(x, y, z, nx, ny);
  const float gpe = fmaf(K.v3, K.dpe_dz[c], fmaf(K.v2, K.dpe_dy[c], K.v1 * K.dpe_dx[c]));
  const float aT = fmaf(K.v3, K.dlnt_dz[c], fmaf(K.v2, K.dlnt_dy[c], K.v1 * K.dlnt_dx[c])) / K.temp[c];
  const float pec = K.pe[c], rpec = 1.0f / pec;
  const float rxpup = up[3], rhou = up[4];
  const float betc = K.beta[p];
  const float t1 = (xx - xxup) * K.rpath;
  const float sgn = copysignf(1.0f, t1);
  const float rxpc = xx * rpec;
  float mc = fmaf(rxpc, gpe, (pec * (rxpc - rxpup)) * K.rpath);
  mc = sgn * fmaxf(0.0f, fminf(sgn * mc, 2.0f * fabsf(t1)));
  const double dt = herm2_clamp((double)fmaf(K.dsup05, xxup + xx, K.dsc2 * (t1 - mc)), K.dtmax);
  const double rdt = __drcp_rn(dt);
  const float rdt4 = (float)rdt;
  float ex, U0, U1, q;
  parab_moments((float)dt, ex, U0, U1, q);
  const float r1mbc = 1.0f / (1.0f - betc);
  const float Bc = betc * r1mbc;
  const float gc = ((K.hknu[f] * r1mbc) * aT) / xx;
  const float rhoc = ss / Bc;
  const float t1s = (ss - ssup) * rdt4;
  const float sgns = copysignf(1.0f, t1s);
  float dsdtau = fmaf(ss, gc, (Bc * (rhoc - rhou)) * rdt4);
  float kf, srem;
  if (sgns * dsdtau <= 0.0f) {
    dsdtau = 0.0f;
    kf = 0.0f;
    srem = 0.0f;
  } else if (sgns * dsdtau >= 2.0f * fabsf(t1s)) {
    dsdtau = 2.0f * t1s;
    kf = 2.0f * rdt4;
    srem = -((2.0f * rdt4) * ssup);
  } else {
    kf = gc + rdt4;
    srem = -((Bc * rhou) * rdt4);
  }
  const double B = __dmul_rn(__dsub_rn(2.0 * (double)U1, (double)q), rdt);
  const double A = __dsub_rn((double)U0, B);
  const float C = q - U1;
  float Inu = fmaf(C, dsdtau, fmaf((float)B, ss, fmaf((float)A, ssup, Inuup * ex)));
  Inu = fmaxf(-Imax, fminf(Imax, Inu));
  work[o + 2 * k1] = Inu;
  if (s.get_psi) {
    const double pl = __dadd_rn(B, __dmul_rn((double)C, (double)kf));
    const float Psi_loc = (float)pl;
    const bool on = dt > 0 && xx > 0 && Psi_loc >= 0.0f && Psi_loc <= 1.0f && fabsf(Inu) < Imax;
    psi[p] = on ? Psi_loc / xx : 0.0f;
    if (s.split_rates) {
      irem[p] = on ? fmaf(C, srem, fmaf((float)A, ssup, Inuup * ex)) : Inu;
      esc[p] = on ? (float)__dsub_rn(1.0, pl) : 1.0f;
    }
  }
}

}  // namespace m3d

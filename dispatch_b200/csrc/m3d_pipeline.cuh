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
                                                           const float *tgx, const float *th2x) {
  extern __shared__ float smem[];
  float *s_tgx = smem, *s_th2x = smem + QLG_NTAB;
  stage_tables(s_tgx, s_th2x, tgx, th2x);
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
      warp_cell_lines(S.L, G, c, s_chi, s_eta, s_x, s_lr, dep, false, false, nullptr, nullptr, nullptr, s_tgx,
                      s_th2x, lane);
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

__device__ __forceinline__ void rot_load(const float *chi, const float *S, size_t plane, int zg, const RotPlane &r, int f,
                                         int x, int y, int nf, int nx, int ny, float &xv, float &sv) {
  const int x1 = wrap(x + r.up1, nx), x2 = x1 + 1 == nx ? 0 : x1 + 1;
  const int y1 = wrap(y + r.up2, ny), y2 = y1 + 1 == ny ? 0 : y1 + 1;
  const size_t o = plane * (size_t)zg + (size_t)f;
  const size_t i11 = o + (size_t)nf * ((size_t)x1 + (size_t)nx * y1), i21 = o + (size_t)nf * ((size_t)x2 + (size_t)nx * y1);
  const size_t i12 = o + (size_t)nf * ((size_t)x1 + (size_t)nx * y2), i22 = o + (size_t)nf * ((size_t)x2 + (size_t)nx * y2);
  float v = r.a * __ldg(chi + i11);
  v = fmaf(r.b, __ldg(chi + i21), v);
  v = fmaf(r.c, __ldg(chi + i12), v);
  xv = fmaf(r.d, __ldg(chi + i22), v);
  float w = r.a * __ldg(S + i11);
  w = fmaf(r.b, __ldg(S + i21), w);
  w = fmaf(r.c, __ldg(S + i12), w);
  sv = fmaf(r.d, __ldg(S + i22), w);
}

// chi, S: (nf, nx, ny, nz) unrotated transfer units of the whole column; rot: per
// global plane; slab_z0: first global plane of each slab (nslab + 1 entries).
__global__ void __launch_bounds__(256) k_quad_rot_column(int nf, int nx, int ny, int nz, const float *chi,
                                                         const float *S, const RotPlane *rot, const int *slab_z0,
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
    rot_load(chi, S, plane, z0, rot[z0], f, x, y, nf, nx, ny, xc, sc);
    rot_load(chi, S, plane, z0 + 1, rot[z0 + 1], f, x, y, nf, nx, ny, xd, sd);
    for (int zl = 1; zl < n; zl++) {
      float Inu, pl;
      quad_step<float>(xu, xc, xd, su, sc, sd, Iu, true, qc.rdsup, qc.dsup1, qc.dsup2, dtmax, Imax, false, Inu, pl);
      Iu = Inu;
      if (zl + 1 < n) {
        xu = xc; su = sc; xc = xd; sc = sd;
        rot_load(chi, S, plane, z0 + zl + 1, rot[z0 + zl + 1], f, x, y, nf, nx, ny, xd, sd);
      }
    }
    float In, pl;
    quad_step<float>(xu, xc, xd, su, sc, sd, Iu, false, qc.rdsup, qc.dsup1, qc.dsup2, dtmax, Imax, false, In, pl);
    gx = xd; gs = sd; gI = In;
  }
  I_top[g] = gI;
}

// save_intensity (rt_patch_mod.f90:4151-4208): ie(f) = <2h nu^5/(c^3 AA) I>_xy
template <typename TI>
__global__ void k_save_intensity(int nf, int ncol, const double *nu, const TI *I_top, float *ie) {
  __shared__ double part[8][33];
  const int f = blockIdx.x * 32 + threadIdx.x;
  double acc = 0.0;
  if (f < nf) {
    const double conv = 2.0 * 6.626176e-27 / (2.99792458e10 * 2.99792458e10 * 2.99792458e10 * 1e8);
    const double n5 = nu[f] * nu[f] * nu[f] * nu[f] * nu[f];
    for (int c = threadIdx.y; c < ncol; c += blockDim.y)
      acc += (double)(float)(conv * n5 * (double)I_top[(size_t)f + (size_t)nf * c]);
  }
  part[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y == 0 && f < nf) {
    double s = 0.0;
    for (int k = 0; k < (int)blockDim.y; k++) s += part[k][threadIdx.x];
    ie[f] = (float)s / (float)ncol;
  }
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

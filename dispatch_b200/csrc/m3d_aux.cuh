// Inputs and bookkeeping around the solvers:
//   update_eta_mask                   SRC/rt_patch_mod.f90:3671-3807
//   compute_lte_populations / lte_pop SRC/atom_mod.f90:1041-1150 (level partition function)
//   add_particle_opacity's per-cell fields: inverse_doppler_factor, compute_vbar2
//   (HOP/ion_mod.f90:198-221) and lnbase (HOP/linelist_mod.f90:1034-1042)
//
// The eta flags are kept dense on the device: eta_src and eta_mask hold one
// byte per (f, cell), eta_gsrc one per (f, x, y) of the upstream ghost plane.
// The reference's sparse rows (eta_row, eta_src(:, row), eta_mask(:, row)) store
// the same flags; the solvers read the dense mask through eta_row(cell) = cell + 1.
#pragma once
#include <cstdint>

namespace m3d {

// q_eta test of one point (update_eta_mask :3722): min(chi, |chi| - q (chi + (1 - beta) chi S)) <= 0
__device__ __forceinline__ bool eta_fire(float chi, float one_m_beta, float S) {
  const float q_eta = 1e-2f;
  return fminf(chi, fabsf(chi) - q_eta * (chi + one_m_beta * chi * S)) <= 0.0f;
}

// new = fire and not src; src |= new.  work is (nf, nx, ny, 0:nz+1, 3).
__global__ void k_eta_fire(int nf, int nx, int ny, int nz, const float *__restrict__ work,
                           const float *__restrict__ beta, uint8_t *__restrict__ src, uint8_t *__restrict__ fresh) {
  const size_t plane = (size_t)nf * nx * ny, n = plane * nz;
  const size_t kplane = plane * (size_t)(nz + 2);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const size_t w = k + plane;  // plane z (1-based) of work
    const float chi = work[w], S = work[w + kplane];
    const bool fire = eta_fire(chi, 1.0f - beta[k], S);
    const bool nw = fire && !src[k];
    if (nw) src[k] = 1;
    fresh[k] = nw;
  }
}

// the upstream ghost plane zg, tested with 1 - beta = 1
__global__ void k_eta_ghost(int nf, int nx, int ny, int nz, int zg, const float *__restrict__ work,
                            uint8_t *__restrict__ gsrc, uint8_t *__restrict__ gfresh) {
  const size_t plane = (size_t)nf * nx * ny;
  const size_t kplane = plane * (size_t)(nz + 2);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < plane; k += (size_t)gridDim.x * blockDim.x) {
    const size_t w = k + plane * (size_t)zg;
    const float chi = work[w], S = work[w + kplane];
    const bool fire = eta_fire(chi, 1.0f, S);
    const bool nw = fire && !gsrc[k];
    if (nw) gsrc[k] = 1;
    gfresh[k] = nw;
  }
}

// mask(f, x, y, z) |= any new flag within rx, ry (periodic) on plane z, on the
// upwind plane z - dir, and (for the slab's first plane z1) on the ghost plane
__global__ void k_eta_spread(int nf, int nx, int ny, int nz, int dir, int rx, int ry, int z1,
                             const uint8_t *__restrict__ fresh, const uint8_t *__restrict__ gfresh,
                             uint8_t *__restrict__ mask) {
  const size_t plane = (size_t)nf * nx * ny, n = plane * nz;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    if (mask[k]) continue;
    const int f = (int)(k % nf);
    const size_t c = k / nf;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((size_t)nx * ny));  // z 0-based
    const int zu = z - dir;
    bool any = false;
    for (int j = -ry; j <= ry && !any; j++) {
      int yy = (y + j) % ny;
      yy = yy < 0 ? yy + ny : yy;
      for (int i = -rx; i <= rx && !any; i++) {
        int xx = (x + i) % nx;
        xx = xx < 0 ? xx + nx : xx;
        const size_t o = (size_t)f + (size_t)nf * ((size_t)xx + (size_t)nx * yy);
        any = fresh[o + plane * (size_t)z] != 0;
        if (!any && zu >= 0 && zu < nz) any = fresh[o + plane * (size_t)zu] != 0;
        if (!any && gfresh && z == z1) any = gfresh[o] != 0;
      }
    }
    if (any) mask[k] = 1;
  }
}

// compute_lte_populations with the level partition function: nstar (ncell, nlevel)
// float64, totn (ncell) in: the element's atoms, out: sum of nstar
__global__ void k_lte_pop(int ncell, int nlevel, const double *__restrict__ g, const double *__restrict__ ev,
                          const int *__restrict__ ion, const float *__restrict__ temp, const float *__restrict__ lsaha,
                          const float *__restrict__ dxi, double *__restrict__ nstar, double *__restrict__ totn) {
  const double E_K = 1.602189e-12 / 1.380662e-16;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const float ekt = (float)(E_K / (double)temp[c]);
    const float dx = dxi ? dxi[c] : 0.0f, ls = lsaha[c];
    double sum = 0.0;
    for (int i = 0; i < nlevel; i++) {
      const int j = ion[i];
      // dxi*0.5*(j-1)*j is real(4) arithmetic, subtracted from the real(8) energy
      const float low = ((dx * 0.5f) * (float)(j - 1)) * (float)j;
      const double evi = ev[i] - (double)low;
      double tns = log(g[i]) - (double)ekt * evi;
      if (j > ion[0]) tns = tns + (double)((float)(j - ion[0]) * ls);
      const double v = exp(tns);
      nstar[(size_t)c + (size_t)ncell * i] = v;
      sum = sum + v;
    }
    const float partition = (float)sum;
    const double tn = totn[c];
    const float norm = (float)(tn / (double)partition);
    double s2 = 0.0;
    for (int i = 0; i < nlevel; i++) {
      double v = (double)norm * nstar[(size_t)c + (size_t)ncell * i];
      if (tn == 0.0) v = 0.0;
      nstar[(size_t)c + (size_t)ncell * i] = v;
      s2 = s2 + v;
    }
    totn[c] = s2;
  }
}

// inverse_doppler_factor, compute_vbar2 and lnbase of one isotope
struct ParticleArgs { double awgt; float vmic; float log_frac; int has_pop_scale; float log_pop_scale; };

__global__ void k_particle_fields(int ncell, ParticleArgs P, const float *__restrict__ temp,
                                  const double *__restrict__ n, const double *__restrict__ part,
                                  float *__restrict__ idf, float *__restrict__ vbar2, float *__restrict__ lnbase) {
  const double BK = 1.380662e-16, UU = 1.6605655e-24, MH = 1.6726e-24, PI = 3.14159265359, CC = 2.99792458e10;
  const float cdop = (float)(2.0 * BK / UU), cvb = (float)(8.0 * BK / (PI * UU)), inv_mh = (float)(UU / MH);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const float T = temp[c];
    float dop = (float)((double)(cdop * T) / P.awgt);
    if (P.vmic > 0.0f) {
      const float vm = P.vmic * 1e5f;
      dop = dop + vm * vm;
    }
    const float id = (float)(CC / (double)sqrtf(dop));
    idf[c] = id;
    vbar2[c] = (float)((double)(cvb * T) * ((double)inv_mh + 1.0 / P.awgt));
    float lb = (float)log(fmax(n[c], DBL_MIN));
    if (P.has_pop_scale) lb = lb + P.log_pop_scale;
    lnbase[c] = (float)((((double)lb - part[c]) + (double)logf(id)) + (double)P.log_frac);
  }
}

}  // namespace m3d

namespace m3d {

// lte_background_emission (rt_patch_mod.f90:2127-2328) with convert_to_work_units
// (:3518-3536), per point: J from the previous iteration (jmode 0), Bnu (1, the
// Planck start) or 0 (2); with PsiJ, the OAB step of scattering preconditioning
// Jali = (J - op Jali_old)/(1 - op), op = sigma PsiJ clamped to [0, op_max], in
// real(8), kept for the next iteration; then eta = chi Bnu + sigma (J - Bnu),
// dJnu = J - Bnu, xhat = chi + eta, ehat = eta/beta.
struct EmissionArgs { int jmode, scat_precond, jali_valid; double op_max; };

__global__ void k_lte_emission(size_t n, EmissionArgs E, const float *__restrict__ chi, const float *__restrict__ sigma,
                               const float *__restrict__ Bnu, const float *__restrict__ beta, const float *__restrict__ J,
                               const float *__restrict__ PsiJ, float *__restrict__ Jali, float *__restrict__ xhat,
                               float *__restrict__ ehat, float *__restrict__ dJnu, unsigned *__restrict__ nneg) {
  unsigned neg = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const float B = Bnu[k];
    float j = E.jmode == 1 ? B : (E.jmode == 2 ? 0.0f : J[k]);
    if (E.jmode == 0 && E.scat_precond) {
      const float sg = sigma ? sigma[k] : 0.0f;
      double op = (double)sg * (double)PsiJ[k];
      op = fmax(0.0, fmin(op, E.op_max));
      const double jfs = (double)j;
      const double jold = E.jali_valid ? (double)Jali[k] : jfs;
      double jn = (jfs - op * jold) / (1.0 - op);
      if (jn < 0.0) { jn = jfs; neg++; }
      j = (float)jn;
      Jali[k] = j;
    }
    const float dj = j - B;
    const float s = sigma ? sigma[k] : 0.0f;
    const float eta = chi[k] * B + s * dj;
    if (dJnu) dJnu[k] = dj;
    xhat[k] = chi[k] + eta;
    ehat[k] = eta / beta[k];
  }
  if (nneg && neg) atomicAdd(nneg, neg);
}

// add_linelist_opacities' last step for line scattering (composition_mod.f90:1864-1874):
// chi_scat in working units to physical extinction, chi_scat *= 1 - beta
__global__ void k_chi_scat_units(size_t n, float *__restrict__ cs, const float *__restrict__ beta) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    cs[k] = cs[k] * (1.0f - beta[k]);
}

}  // namespace m3d

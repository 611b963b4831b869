// Columns of uneven depth for the batched 1.5D ALI: the per-point arrays hold
// the cells of every column back to back (column c owns cells col_off[c] ..
// col_off[c+1]-1, bottom to top), frequency fastest.
#pragma once
#include "m3d_kernels.cuh"

namespace m3d {

struct ColArgs {
  int nf, ncol;
  const int *col_off;
  const double *dz;
  double mu;          // direction cosine: > 0 upwards, < 0 downwards
  int bottom;         // ghost of an upward ray: 1 zero, 2 the PCHIP extrapolation
  float dtau_max, Inu_max;
};

// long_char_linear (rt_solvers_mod.f90:666-757) along each column, one thread per
// (column, f), with the upstream ghost of set_upstream_boundary folded in: zero
// at the top for downward rays; at the bottom either zero or the PCHIP
// extrapolation from the first two cells with I = S (k_upstream_boundary, mode 2).
// chi, S are the transfer units; inu, psi, irem, esc receive the solution.
__global__ void k_long_char_columns(ColArgs A, PchipConst pc, const float *__restrict__ chi,
                                    const float *__restrict__ S, float *__restrict__ inu, float *__restrict__ psi,
                                    float *__restrict__ irem, float *__restrict__ esc, float *__restrict__ Jnu,
                                    float *__restrict__ PsiJ, float wmu) {
  // with Jnu, the epilogue of integrate_intensity (rt_patch_mod.f90:3399-3431) too
  const float w2 = 2.0f * wmu;
  const size_t nf = (size_t)A.nf;
  const size_t n = nf * A.ncol;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(g % nf), c = (int)(g / nf);
    const int k0 = A.col_off[c], k1 = A.col_off[c + 1], nz = k1 - k0;
    if (nz < 1) continue;
    const int dir = A.mu > 0 ? 1 : -1;
    const float ds = (float)A.dz[c];
    const float dsup05 = (float)((double)(0.5f * ds) / fabs(A.mu));
    float xxup = 0.0f, ssup = 0.0f, Inuup = 0.0f;
    if (dir > 0 && A.bottom == 2 && nz >= 2) {
      const size_t p1 = f + nf * k0, p2 = f + nf * (k0 + 1);
      float gv[2];
      const float y1s[2] = {chi[p1], S[p1]}, y2s[2] = {chi[p2], S[p2]};
      for (int k = 0; k < 2; k++) {
        const float y1 = y1s[k], y2 = y2s[k];
        const float dy1 = y2 - y1;
        const float dydx1 = (2.0f * dy1) / pc.dx1 - 0.0f;
        const float v = (pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * dydx1 + pc.cm1 * 0.0f);
        gv[k] = fmaxf(v, 0.0f);
      }
      xxup = gv[0];
      ssup = gv[1];
      Inuup = ssup;
    }
    const float dtmax = -A.dtau_max, Imax = A.Inu_max;
    for (int i = 0; i < nz; i++) {
      const int cell = dir > 0 ? k0 + i : k1 - 1 - i;
      const size_t o = f + nf * cell;
      const float xx = chi[o], ss = S[o];
      float dt = dsup05 * (xxup + xx);
      dt = fmaxf(dt, dtmax);
      float E, W, Psi, Esc;
      linear_weights(dt, E, W, Psi, Esc);
      float Inu = fma_t(Psi, ss, fma_t(W, ssup, Inuup * E));
      const bool off = dt <= 0 || xx <= 0 || fabsf(Inu) > Imax;
      const float Irem = fma_t(W, ssup, Inuup * E);
      Inu = fmaxf(-Imax, fminf(Imax, Inu));
      Psi = off ? 0.0f : Psi;
      irem[o] = off ? Inu : Irem;
      esc[o] = off ? 1.0f : Esc;
      inu[o] = Inu;
      const float ps = (dt > 0 && xx > 0) ? Psi / xx : 0.0f;
      psi[o] = ps;
      if (Jnu) {
        Jnu[o] = fmaf(w2, Inu, Jnu[o]);
        PsiJ[o] = fmaf(w2, ps, PsiJ[o]);
      }
      xxup = xx;
      ssup = ss;
      Inuup = Inu;
    }
  }
}

// dst(f, cell) = src(cell): the grey continuum on a window's frequencies
__global__ void k_broadcast_cells(size_t n, int nf, const float *__restrict__ src, float *__restrict__ dst) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    dst[k] = src[k / nf];
}

// vproj = vz * mu in real(4), as get_vproj forms it for a vertical velocity
__global__ void k_scale_cells(int n, const float *__restrict__ vz, float mu, float *__restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) out[k] = vz[k] * mu;
}

}  // namespace m3d

// Sampled opacity tables (HOP/optab_mod.f90): a background or line-list opacity
// per unit chi500 tabulated on (wavelength, PC axis 1, PC axis 2) of (ln T, ln ne),
// sampled per (frequency, cell) by a separable tensor-product cubic Hermite with
// precomputed node slopes.
//
// Device layout: one float4 per node (val, dl, dt, de) -- the value and its slopes
// along the wavelength and the two PC axes -- wavelength fastest, so one 16-byte
// load brings everything the collapse needs from a node and the frequencies of a
// window read a contiguous run of nodes.  A second array holds the scattering
// component.  The window's slice of the table (the nodes its frequencies bracket,
// at every (it, je)) stays in L2 while the cells stream through.
#pragma once
#include "m3d_kernels.cuh"

namespace m3d {

struct OptabDev {
  int nnu, ntemp, nne, has_scat;
  const double *lam;
  const float4 *tv, *ts;
  double mu0, mu1, r11, r21, r12, r22, c01, c02, dc1, dc2;
};

// per-frequency bracket on the wavelength nodes: cnt = number of nodes below the
// query, k the 0-based interval, and hermite_coefs of the position in it; node is
// the wavelength node the query sits on (the interval's end with weights 0 and 1
// and vanishing slope weights) or -1
struct OptabFreq {
  int k, cnt;
  float pl, wc0, wc1, wcm0, wcm1;
  int node;
};

// A query on a node: the weights are (c0, c1) = (1, 0) or (0, 1) and cm0 = cm1 = 0,
// so each term the collapse forms from the other node is a product with an exact
// zero and it returns the node's own value and PC slopes.  The node's float4 alone
// then gives the same result for finite tables (a -0 can come out as +0).
__device__ __forceinline__ int optab_on_node(const float c[5], int k) {
  if (c[3] != 0.0f || c[4] != 0.0f) return -1;
  if (c[1] == 1.0f && c[2] == 0.0f) return k;
  if (c[1] == 0.0f && c[2] == 1.0f) return k + 1;
  return -1;
}

// hermite_coefs (interpol_mod.f90:171-188): p, c0, c1, cm0, cm1
__host__ __device__ __forceinline__ void optab_hcoefs(float t, float h, float c[5]) {
  const float t2 = t * t, t3 = t2 * t;
  const float p = 3.0f * t2 - 2.0f * t3;
  c[0] = p;
  c[1] = 1.0f - p;
  c[2] = p;
  c[3] = h * ((t3 - 2.0f * t2) + t);
  c[4] = h * (t3 - t2);
}

// the bracket of optab_mod.f90:214/358 from the count of nodes below x:
// k = min(max(searchsorted, 1), nnu - 1) is that count clamped to [1, nnu - 1]
__device__ __forceinline__ int optab_interval(int nnu, const double *lam, int cnt, double x, float c[5]) {
  int k = cnt < 1 ? 1 : (cnt > nnu - 1 ? nnu - 1 : cnt);
  k -= 1;
  const double l0 = lam[k], l1 = lam[k + 1];
  optab_hcoefs((float)((x - l0) / (l1 - l0)), (float)(l1 - l0), c);
  return k;
}

__global__ void k_optab_freq(int nf, const double *lam_q, int nnu, const double *lam, OptabFreq *fc) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const double x = lam_q[f];
  int lo = 0, hi = nnu;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (lam[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  float c[5];
  OptabFreq o;
  o.cnt = lo;
  o.k = optab_interval(nnu, lam, lo, x, c);
  o.pl = c[0];
  o.wc0 = c[1];
  o.wc1 = c[2];
  o.wcm0 = c[3];
  o.wcm1 = c[4];
  o.node = optab_on_node(c, o.k);
  fc[f] = o;
}

// the cell's PC coordinates and Hermite coefficients (optab_mod.f90:225-238)
__device__ __forceinline__ void optab_cell(const OptabDev &T, double temp, double ne, int &it, int &je, float tc[5],
                                           float nc[5]) {
  const double d1 = log(temp) - T.mu0;
  const double d2 = log(ne) - T.mu1;
  const double p1 = __dadd_rn(__dmul_rn(T.r11, d1), __dmul_rn(T.r21, d2));
  const double p2 = __dadd_rn(__dmul_rn(T.r12, d1), __dmul_rn(T.r22, d2));
  const double ft = __dadd_rn(__dmul_rn(p1 - T.c01, __drcp_rn(T.dc1)), 1.0);
  const double fe = __dadd_rn(__dmul_rn(p2 - T.c02, __drcp_rn(T.dc2)), 1.0);
  const double ift = fmin(fmax(floor(ft), 1.0), (double)(T.ntemp - 1));
  const double ife = fmin(fmax(floor(fe), 1.0), (double)(T.nne - 1));
  optab_hcoefs((float)(ft - ift), (float)T.dc1, tc);
  optab_hcoefs((float)(fe - ife), (float)T.dc2, nc);
  it = (int)ift - 1;
  je = (int)ife - 1;
}

// collapse (optab_mod.f90:251-286): wavelength at the four (temp, ne) corners,
// the PC slopes carried across it, then temp, then ne
__device__ __forceinline__ float optab_collapse(const float4 *t, size_t base, size_t sit, size_t sje, const float w[5],
                                                const float tc[5], const float nc[5]) {
  const float pl = w[0], opl = 1.0f - pl;
  float v[4], gt[4], ge[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const size_t a = base + (c & 1) * sit + (c >> 1) * sje;
    const float4 A = __ldg(t + a), B = __ldg(t + a + 1);
    v[c] = fmaf(w[4], B.y, fmaf(w[3], A.y, fmaf(w[2], B.x, w[1] * A.x)));
    gt[c] = fmaf(pl, B.z, opl * A.z);
    ge[c] = fmaf(pl, B.w, opl * A.w);
  }
  const float pt = tc[0], opt = 1.0f - pt;
  const float f0 = fmaf(tc[4], gt[1], fmaf(tc[3], gt[0], fmaf(tc[2], v[1], tc[1] * v[0])));
  const float f1 = fmaf(tc[4], gt[3], fmaf(tc[3], gt[2], fmaf(tc[2], v[3], tc[1] * v[2])));
  const float ge0 = fmaf(pt, ge[1], opt * ge[0]);
  const float ge1 = fmaf(pt, ge[3], opt * ge[2]);
  return fmaf(nc[4], ge1, fmaf(nc[3], ge0, fmaf(nc[2], f1, nc[1] * f0)));
}

// the collapse of a query on node n: the node's value and PC slopes at the four
// (temp, ne) corners, then temp, then ne, as optab_collapse forms them
__device__ __forceinline__ float optab_collapse_node(const float4 *t, size_t base, size_t sit, size_t sje,
                                                     const float tc[5], const float nc[5]) {
  float v[4], gt[4], ge[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const float4 A = __ldg(t + base + (c & 1) * sit + (c >> 1) * sje);
    v[c] = A.x;
    gt[c] = A.z;
    ge[c] = A.w;
  }
  const float pt = tc[0], opt = 1.0f - pt;
  const float f0 = fmaf(tc[4], gt[1], fmaf(tc[3], gt[0], fmaf(tc[2], v[1], tc[1] * v[0])));
  const float f1 = fmaf(tc[4], gt[3], fmaf(tc[3], gt[2], fmaf(tc[2], v[3], tc[1] * v[2])));
  const float ge0 = fmaf(pt, ge[1], opt * ge[0]);
  const float ge1 = fmaf(pt, ge[3], opt * ge[2]);
  return fmaf(nc[4], ge1, fmaf(nc[3], ge0, fmaf(nc[2], f1, nc[1] * f0)));
}

constexpr int kOptabWarps = 8;
// both samplers are latency-bound: at most 64 registers give 4 blocks (32 warps) per
// SM, measured faster than 66-77 registers at 3 blocks and than 48 or 40 with spills
constexpr int kOptabMinBlocks = 4;
constexpr int kOptabUnroll = 1;   // frequencies per lane per pass of sample_interpolate_ll
constexpr int kOptabLLMinBlocks = 4;   // 5 or 6 spill and are slower

// sample_interpolate (optab_mod.f90:181-287): one warp per cell, lanes over the
// frequencies; back = (kappa + kappa_scat) chi500, scat = kappa_scat chi500
__global__ void __launch_bounds__(32 * kOptabWarps, kOptabMinBlocks) k_optab_sample(OptabDev T, int nf, long long ncell,
                                                                   const double *temp, const double *ne,
                                                                   const float *chi500, const OptabFreq *fc,
                                                                   float *back, float *scat) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (long long)blockIdx.x * kOptabWarps + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * kOptabWarps;
  const size_t sit = (size_t)T.nnu, sje = (size_t)T.nnu * T.ntemp;
  for (long long c = w0; c < ncell; c += nw) {
    int it, je;
    float tc[5], nc[5];
    optab_cell(T, temp[c], ne[c], it, je, tc, nc);
    const float ch = chi500[c];
    const size_t cb = (size_t)it * sit + (size_t)je * sje;
    for (int f = lane; f < nf; f += 32) {
      const OptabFreq q = fc[f];
      float kap, kas;
      if (q.node >= 0) {
        kap = optab_collapse_node(T.tv, cb + q.node, sit, sje, tc, nc);
        kas = optab_collapse_node(T.ts, cb + q.node, sit, sje, tc, nc);
      } else {
        const float w[5] = {q.pl, q.wc0, q.wc1, q.wcm0, q.wcm1};
        kap = optab_collapse(T.tv, cb + q.k, sit, sje, w, tc, nc);
        kas = optab_collapse(T.ts, cb + q.k, sit, sje, w, tc, nc);
      }
      const size_t o = (size_t)c * nf + f;
      back[o] = (kap + kas) * ch;
      scat[o] = kas * ch;
    }
  }
}

// sample_interpolate_ll (optab_mod.f90:300-409): the query wavelength of each
// cell is lam_q (1 + vproj), bracketed by walking from the unshifted count;
// xhat, ehat += kappa chi500, and chi_scat += kappa_scat chi500 when given.
// A lane takes kOptabUnroll frequencies per pass: their work slots are read and
// their brackets found before the table lookups.  One frequency at 4 blocks per SM
// measured faster (8.7 ms at 2.1 M cells x 256) than two (10.6 ms), which held the
// reads of two in flight at the cost of registers.
__global__ void __launch_bounds__(32 * kOptabWarps, kOptabLLMinBlocks) k_optab_sample_ll(OptabDev T, int nf, long long ncell,
                                                                      const double *temp, const double *ne,
                                                                      const float *chi500, const float *vproj,
                                                                      const double *lam_q, const OptabFreq *fc,
                                                                      float *xhat, float *ehat, float *chi_scat) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (long long)blockIdx.x * kOptabWarps + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * kOptabWarps;
  const size_t sit = (size_t)T.nnu, sje = (size_t)T.nnu * T.ntemp;
  const int nnu = T.nnu;
  const double *lam = T.lam;
  for (long long c = w0; c < ncell; c += nw) {
    int it, je;
    float tc[5], nc[5];
    optab_cell(T, temp[c], ne[c], it, je, tc, nc);
    const float ch = chi500[c];
    const double vf = 1.0 + (double)vproj[c];
    const size_t cb = (size_t)it * sit + (size_t)je * sje;
    for (int f0 = lane; f0 < nf; f0 += 32 * kOptabUnroll) {
      float xv[kOptabUnroll], ev[kOptabUnroll], sv[kOptabUnroll];
      int k[kOptabUnroll], nd[kOptabUnroll];
      float w[kOptabUnroll][5];
#pragma unroll
      for (int u = 0; u < kOptabUnroll; u++) {
        const int f = f0 + 32 * u;
        if (f >= nf) break;
        const size_t o = (size_t)c * nf + f;
        xv[u] = xhat[o];
        ev[u] = ehat[o];
        if (chi_scat) sv[u] = chi_scat[o];
        const double x = __dmul_rn(lam_q[f], vf);
        int cnt = fc[f].cnt;
        while (cnt < nnu && lam[cnt] < x) cnt++;
        while (cnt > 0 && lam[cnt - 1] >= x) cnt--;
        k[u] = optab_interval(nnu, lam, cnt, x, w[u]);
        nd[u] = optab_on_node(w[u], k[u]);
      }
#pragma unroll
      for (int u = 0; u < kOptabUnroll; u++) {
        const int f = f0 + 32 * u;
        if (f >= nf) break;
        const float kap = nd[u] >= 0 ? optab_collapse_node(T.tv, cb + nd[u], sit, sje, tc, nc)
                                     : optab_collapse(T.tv, cb + k[u], sit, sje, w[u], tc, nc);
        const float add = kap * ch;
        xv[u] = xv[u] + add;
        ev[u] = ev[u] + add;
        if (chi_scat) {
          const float kas = nd[u] >= 0 ? optab_collapse_node(T.ts, cb + nd[u], sit, sje, tc, nc)
                                       : optab_collapse(T.ts, cb + k[u], sit, sje, w[u], tc, nc);
          sv[u] = sv[u] + kas * ch;
        }
      }
#pragma unroll
      for (int u = 0; u < kOptabUnroll; u++) {
        const int f = f0 + 32 * u;
        if (f >= nf) break;
        const size_t o = (size_t)c * nf + f;
        xhat[o] = xv[u];
        ehat[o] = ev[u];
        if (chi_scat) chi_scat[o] = sv[u];
      }
    }
  }
}

// sample_build_derivatives (optab_mod.f90:125-166), one thread per node.
// pchip_slopes8 (interpol_mod.f90:240-284) along the fp64 wavelength nodes:
// the interior slope of node i of a line y (stride 1)
__device__ __forceinline__ double pchip8_interior(const double *x, const float *y, int i) {
  const double dxm = x[i] - x[i - 1], dxp = x[i + 1] - x[i];
  const double dym = (double)y[i] - (double)y[i - 1], dyp = (double)y[i + 1] - (double)y[i];
  if (dym == 0 || dyp == 0) return 0.0;
  const double d1 = dym / dxm, d2 = dyp / dxp;
  if (copysign(1.0, d1) != copysign(1.0, d2)) return 0.0;
  const double alpha = (1.0 + dxm / (dxp + dxm)) / 3.0;
  return 1.0 / ((1.0 - alpha) / d1 + alpha / d2);
}

__global__ void k_optab_lam_slopes(int nnu, long long nlines, const double *lam, const float *val, float *dl) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= (size_t)nnu * nlines) return;
  const int k = (int)(g % nnu);
  const float *y = val + (g - k);
  double s;
  if (nnu == 2) {
    const double dy = (double)y[1] - (double)y[0], dx = lam[1] - lam[0];
    const double a = 2.0 * dy / dx - dy / dx;
    s = k == 0 ? a : 2.0 * dy / dx - a;
  } else if (k == 0) {
    s = 2.0 * ((double)y[1] - (double)y[0]) / (lam[1] - lam[0]) - pchip8_interior(lam, y, 1);
  } else if (k == nnu - 1) {
    s = 2.0 * ((double)y[k] - (double)y[k - 1]) / (lam[k] - lam[k - 1]) - pchip8_interior(lam, y, k - 1);
  } else {
    s = pchip8_interior(lam, y, k);
  }
  dl[g] = (float)s;
}

// pchip_slopes4 (interpol_mod.f90:193-235) along a regular PC axis, the node
// slopes pchip_mono4 returns at the nodes (:335-362): node i of a line of n
// nodes at stride st; the axis node i is (float)(c0 + i dc)
__device__ __forceinline__ float pchip4_interior(double c0, double dc, const float *y, size_t st, int i) {
  const float xm = (float)(c0 + (double)(i - 1) * dc), x0 = (float)(c0 + (double)i * dc);
  const float xp = (float)(c0 + (double)(i + 1) * dc);
  const float dxm = x0 - xm, dxp = xp - x0;
  const float dym = y[i * st] - y[(i - 1) * st], dyp = y[(i + 1) * st] - y[i * st];
  if (dym == 0 || dyp == 0) return 0.0f;
  const double d1 = (double)(dym / dxm), d2 = (double)(dyp / dxp);
  if (copysign(1.0, d1) != copysign(1.0, d2)) return 0.0f;
  const double alpha = (double)((1.0f + dxm / (dxp + dxm)) / 3.0f);
  return (float)(1.0 / ((1.0 - alpha) / d1 + alpha / d2));
}

__global__ void k_optab_axis_slopes(int nnu, int ntemp, int nne, int dim, double c0, double dc, const float *val,
                                    float *out) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= (size_t)nnu * ntemp * nne) return;
  const int it = (int)((g / nnu) % ntemp), je = (int)(g / ((size_t)nnu * ntemp));
  const int n = dim == 1 ? ntemp : nne;
  const int i = dim == 1 ? it : je;
  const size_t st = dim == 1 ? (size_t)nnu : (size_t)nnu * ntemp;
  const float *y = val + (g - (size_t)i * st);
  auto ax = [&](int j) { return (float)(c0 + (double)j * dc); };
  float s;
  if (n == 2) {
    const float dy = y[st] - y[0], dx = ax(1) - ax(0);
    const float a = 2.0f * dy / dx - dy / dx;
    s = i == 0 ? a : 2.0f * dy / dx - a;
  } else if (i == 0) {
    s = 2.0f * (y[st] - y[0]) / (ax(1) - ax(0)) - pchip4_interior(c0, dc, y, st, 1);
  } else if (i == n - 1) {
    s = 2.0f * (y[i * st] - y[(i - 1) * st]) / (ax(i) - ax(i - 1)) - pchip4_interior(c0, dc, y, st, i - 1);
  } else {
    s = pchip4_interior(c0, dc, y, st, i);
  }
  out[g] = s;
}

__global__ void k_optab_pack(size_t n, const float *val, const float *dl, const float *dt, const float *de,
                             float4 *t) {
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g < n) t[g] = make_float4(val[g], dl[g], dt[g], de[g]);
}

}  // namespace m3d

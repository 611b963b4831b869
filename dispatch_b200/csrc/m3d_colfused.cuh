// The fused column sweep of the batched 1.5D ALI: one launch per window and
// hemisphere runs, for every column and every direction of the hemisphere,
//   add_bound_bound_opacities with the split tracking   SRC/rt_patch_mod.f90:2689-2831, 3150-3187
//   work_to_transfer_units (split form)                 SRC/rt_patch_mod.f90:3571-3651
//   long_char_linear with the upstream ghost            SRC/rt_solvers_mod.f90:666-757, rt_patch_mod.f90:3270-3393
//   integrate_intensity                                 SRC/rt_patch_mod.f90:3399-3431
//   bound_bound_rates ('largest', per direction)        SRC/rt_patch_mod.f90:2852-3142
// with the per-point values in registers: a point's opacity, transfer units,
// intensity and rate terms are formed where the sweep reaches it, and only the
// window's inputs (xhat, ehat, beta, Bnu), J/PsiJ and the per-(line, cell) rates
// touch global memory.  The arithmetic is that of k_bb_opacity, k_long_char_columns
// and k_bb_rates term for term, so the results are theirs bit for bit.
//
// One CTA owns one column; its threads run along frequency and walk the column in
// chunks of zchunk cells.  Per chunk the CTA stages every (cell, line) constant
// once (the QLG-bot set-up of the line's damping, Rij b_j, Rij b_i and 1/n_ref).
// A point's inputs are read once for all the launch's directions, which then run in
// turn, each with its own upstream state; each direction's rate terms go to its own
// shared row per cell, and at the chunk's end one thread per (line, cell) adds the
// line's terms in ascending f -- bound_bound_rates' order -- for each direction in
// turn and updates the rates.
#pragma once
#include "m3d_columns.cuh"
#include "m3d_nlte.cuh"

namespace m3d {

constexpr int kColFusedMaxDir = 16;   // directions of one launch (a hemisphere's group)
constexpr int kColFusedMaxLines = 4;  // lines whose window holds one frequency
constexpr int kColFusedConsts = 8;    // per (cell, line): ih, bL, gG, cZH, cL2, Rij bj, Rij bi, 1/n_ref
constexpr int kColFusedLineInts = 8;  // per line: slot offset, blue, index, kind, length

struct ColFusedArgs {
  NlWinDev W;
  int ncell, nslot, rs, zchunk, nd, first, precond, bottom;
  const int *col_off, *soff;
  const double *dz;
  double mu[kColFusedMaxDir];
  float wmu[kColFusedMaxDir];
  PchipConst pc;
  float dtau_max, Inu_max, units_floor, wtot;
  const double *b, *nstar, *pop_ratio, *e_kT;
  const float *inv_df, *vz, *adamp;
  const float2 *tab;
  const float *xhat, *ehat, *beta, *Bnu;
  float *J, *PsiJ, *gw_ij, *gw_ji;
};

// shared-memory bytes of one CTA
__host__ __device__ inline size_t col_fused_smem(int nf, int nline, int nslot, int rs, int zchunk, int nd) {
  const size_t nfl = 3 * (size_t)nd * zchunk * rs + (size_t)zchunk * nline * kColFusedConsts + 2 * (size_t)zchunk +
                     (2 + (size_t)nd) * nslot + 3 * (size_t)nd * nf + 3 * (size_t)nd;
  const size_t nint = (size_t)nline * kColFusedLineInts + (nf + 1) + (size_t)nslot;
  return 4 * (nfl + nint);
}

// the constants of line i in cell c: the profile's QLG-bot set-up (qlg_bot_profile,
// qlg_mod.f90:682-689), k_bb_opacity's Rij bj and Rij bi (= k_bb_rates' eta_coef and
// abs_coef, formed the same way) and k_bb_rates' 1/n_ref
__device__ __forceinline__ void colf_line_consts(const ColFusedArgs &A, int i, int c, float *out) {
  const NlWinDev &W = A.W;
  const size_t nc = (size_t)A.ncell;
  const int li = W.li[i], lj = W.lj[i];
  const double nsi = A.nstar[(size_t)c + nc * li], nsj = A.nstar[(size_t)c + nc * lj];
  const float ekt = (float)A.e_kT[c];
  const float ni = (float)(nsi * A.pop_ratio[c]);
  float bi = (float)A.b[(size_t)c + nc * li], bj = (float)A.b[(size_t)c + nc * lj];
  const float lower_off = (float)(W.lower_ev[i] - W.ev[li]);
  if (lower_off != 0.0f) {
    bi = bi * expf(-lower_off * ekt);
    bj = bj * expf(-lower_off * ekt);
  }
  const float Rij = (float)((double)ni * W.Bij[i]);
  float inr = 0.0f;
  if (nsi > 0 && nsj > 0) {
    const double beta_ref = nsj * W.g[li] / (nsi * W.g[lj]);
    inr = (float)fmin((1.0 - beta_ref) / beta_ref, 1e35);
  }
  const QlgCoef q = qlg_setup(A.adamp[(size_t)c + nc * i], 1.0f, 0.8325546112f, 1.7724538509f);
  out[0] = q.ih;
  out[1] = q.bL;
  out[2] = q.gG;
  out[3] = q.cZH;
  out[4] = q.cL2;
  out[5] = Rij * bj;
  out[6] = Rij * bi;
  out[7] = inr;
}

// one point's line opacity with the split tracking, then its transfer units
// (k_bb_opacity with the units epilogue); phi keeps the lines' profiles
struct ColfPoint {
  float chi, S, oL, oR, cL, cR;
  int oid, cid;
  float phi[kColFusedMaxLines];
};

__device__ __forceinline__ void colf_opacity(const ColFusedArgs &A, const float *Cz, const int *sLi, const int *sLx,
                                             const float *sq, int f, int p0, int n, float vpr, float idf, float xh,
                                             float eh, float be, ColfPoint &P) {
  P.oL = eh;
  P.oR = 0.0f;
  P.cL = xh;
  P.cR = 0.0f;
  P.oid = 0;
  P.cid = 0;
#pragma unroll
  for (int k = 0; k < kColFusedMaxLines; k++) {
    P.phi[k] = 0.0f;
    if (k < n) {
      const int i = sLx[p0 + k];
      const int *Li = sLi + kColFusedLineInts * i;
      const float *C = Cz + kColFusedConsts * i;
      const float q = sq[Li[0] + f - Li[1]];
      const QlgCoef c{C[0], C[1], C[2], C[3], C[4]};
      const float v = fabsf(q - vpr) * idf;
      const bool mk = __all_sync(__activemask(), v * c.ih <= 4611686018427387904.0f);
      const float K1 = mk ? qlg_eval<true>(A.tab, c, v) : qlg_eval<false>(A.tab, c, v);
      const float phi = ((K1 * 0.5641895835f) * idf) * (q + 1.0f);
      P.phi[k] = phi;
      xh = xh + phi * C[6];
      eh = eh + phi * C[5];
      add_largest(phi * C[5], Li[2], P.oL, P.oR, P.oid);
      add_largest(phi * C[6], Li[2], P.cL, P.cR, P.cid);
    }
  }
  units_split_point(xh, be, P.oL, P.oR, 0.0f, false, A.units_floor, 0, P.chi, P.S);
}

// the upstream ghost of direction d at frequency f: zero, or for upward rays the
// PCHIP extrapolation from the first two cells' transfer units with I = S
// (k_long_char_columns); the first chunk holds the first two cells' constants
__device__ __forceinline__ void colf_ghost(const ColFusedArgs &A, const float *sC, const float *sVz,
                                           const float *sIdf, const int *sLi, const int *sLx, const float *sq,
                                           int nl, int f, int p0, int n, int k0, float muf, float &xu, float &su,
                                           float &iu) {
  const size_t nfs = (size_t)A.W.nf;
  ColfPoint P1, P2;
  const size_t o1 = f + nfs * k0, o2 = f + nfs * (k0 + 1);
  colf_opacity(A, sC, sLi, sLx, sq, f, p0, n, sVz[0] * muf, sIdf[0], A.xhat[o1], A.ehat[o1], A.beta[o1], P1);
  colf_opacity(A, sC + (size_t)nl * kColFusedConsts, sLi, sLx, sq, f, p0, n, sVz[1] * muf, sIdf[1], A.xhat[o2],
               A.ehat[o2], A.beta[o2], P2);
  const PchipConst pc = A.pc;
  float gv[2];
  const float y1s[2] = {P1.chi, P1.S}, y2s[2] = {P2.chi, P2.S};
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const float y1 = y1s[k], y2 = y2s[k];
    const float dy1 = y2 - y1;
    const float dydx1 = (2.0f * dy1) / pc.dx1 - 0.0f;
    const float v = (pc.c0 * y1 + pc.p * y2) + pc.dx1 * (pc.cm0 * dydx1 + pc.cm1 * 0.0f);
    gv[k] = fmaxf(v, 0.0f);
  }
  xu = gv[0];
  su = gv[1];
  iu = su;
}

// a point's inputs, read once per hemisphere (streaming loads: the QLG table keeps L1)
__device__ __forceinline__ void colf_load(const ColFusedArgs &A, size_t o, float &xh, float &eh, float &be,
                                          float &nb, float &Jv, float &Pv) {
  xh = __ldcs(A.xhat + o);
  eh = __ldcs(A.ehat + o);
  be = __ldcs(A.beta + o);
  nb = __ldcs(A.Bnu + o);
  Jv = A.first ? 0.0f : __ldcs(A.J + o);
  Pv = A.first ? 0.0f : __ldcs(A.PsiJ + o);
}

// Every direction of the launch at one point: the point's inputs and J/PsiJ are read
// once, the directions run in turn (each its own upstream state), J and PsiJ add
// the directions in order, and each direction's rate terms go to its own rows.
__global__ void __launch_bounds__(256, 4) k_col_ali_fused(ColFusedArgs A) {
  extern __shared__ float sm[];
  const NlWinDev &W = A.W;
  const int nf = W.nf, nl = W.nline, Z = A.zchunk, RS = A.rs, NS = A.nslot, ND = A.nd;
  const int BS = blockDim.x, tid = threadIdx.x;
  const size_t ZR = (size_t)Z * RS;
  float *sT = sm;                                          // (ND, 3, Z, RS) rate terms t0, t1, t3
  float *sC = sT + (size_t)ND * 3 * ZR;                    // (Z, nl, 8)
  float *sVz = sC + (size_t)Z * nl * kColFusedConsts;      // (Z)
  float *sIdf = sVz + Z;                                   // (Z)
  float *sq = sIdf + Z;                                    // (NS) q of each line point
  float *swq = sq + NS;                                    // (NS) profile weights
  float *swm = swq + NS;                                   // (ND, NS) wmu wnu Aij
  float *sXu = swm + (size_t)ND * NS;                      // (ND, nf) upstream chi, S, I
  float *sSu = sXu + (size_t)ND * nf;
  float *sIu = sSu + (size_t)ND * nf;
  float *sDir = sIu + (size_t)ND * nf;                     // (ND, 3): mu, ds/2|mu|, 2 wmu
  int *sLi = reinterpret_cast<int *>(sDir + 3 * ND);       // (nl, 8)
  int *sLp = sLi + (size_t)kColFusedLineInts * nl;         // (nf + 1) per-frequency line lists
  int *sLx = sLp + nf + 1;                                 // (NS)

  const int col = blockIdx.x;
  const int k0 = A.col_off[col], k1 = A.col_off[col + 1], nz = k1 - k0;
  const size_t nfs = (size_t)nf;
  const float ds = (float)A.dz[col];
  for (int i = tid; i < nl; i += BS) {
    const bool act = !W.lactive || W.lactive[i];
    int *Li = sLi + kColFusedLineInts * i;
    Li[0] = A.soff[i];
    Li[1] = W.lblue[i];
    Li[2] = W.lindex[i];
    Li[3] = act ? (W.lsums[i] ? 1 : 2) : 0;  // 2: the line normalises its own profile
    Li[4] = W.lred[i] - W.lblue[i] + 1;
  }
  for (int f = tid; f <= nf; f += BS) sLp[f] = W.lf_ptr[f];
  for (int p = tid; p < NS; p += BS) sLx[p] = W.lf_idx[p];
  for (int f = tid; f < nf; f += BS) {
    for (int p = W.lf_ptr[f]; p < W.lf_ptr[f + 1]; p++) {
      const int i = W.lf_idx[p];
      const int o = W.loff[i] + f - W.lblue[i], s = A.soff[i] + f - W.lblue[i];
      sq[s] = W.q[o];
      swq[s] = (float)W.wq[o];
      for (int d = 0; d < ND; d++) swm[(size_t)d * NS + s] = (float)((double)A.wmu[d] * W.wnu[o] * W.Aij[i]);
    }
  }
  for (int d = tid; d < ND; d += BS) {
    sDir[3 * d] = (float)A.mu[d];
    sDir[3 * d + 1] = (float)((double)(0.5f * ds) / fabs(A.mu[d]));
    sDir[3 * d + 2] = 2.0f * A.wmu[d];
  }
  const int dir = A.mu[0] > 0 ? 1 : -1;
  const float dtmax = -A.dtau_max, Imax = A.Inu_max;

  for (int i0 = 0; i0 < nz; i0 += Z) {
    const int zc = min(Z, nz - i0);
    __syncthreads();  // the tables above, or the previous chunk's sums
    for (int p = tid; p < nl * zc; p += BS) {
      const int i = p / zc, zz = p - i * zc;
      if (!sLi[kColFusedLineInts * i + 3]) continue;
      const int c = dir > 0 ? k0 + i0 + zz : k1 - 1 - (i0 + zz);
      colf_line_consts(A, i, c, sC + ((size_t)zz * nl + i) * kColFusedConsts);
    }
    for (int zz = tid; zz < zc; zz += BS) {
      const int c = dir > 0 ? k0 + i0 + zz : k1 - 1 - (i0 + zz);
      sVz[zz] = A.vz[c];
      sIdf[zz] = A.inv_df[c];
    }
    __syncthreads();
    if (i0 == 0) {
      for (int f = tid; f < nf; f += BS) {
        const int p0 = sLp[f], n = sLp[f + 1] - p0;
        for (int d = 0; d < ND; d++) {
          float xu = 0.0f, su = 0.0f, iu = 0.0f;
          if (dir > 0 && A.bottom == 2 && nz >= 2)
            colf_ghost(A, sC, sVz, sIdf, sLi, sLx, sq, nl, f, p0, n, k0, sDir[3 * d], xu, su, iu);
          sXu[(size_t)d * nf + f] = xu;
          sSu[(size_t)d * nf + f] = su;
          sIu[(size_t)d * nf + f] = iu;
        }
      }
    }
    // the thread's points of the chunk, cells outer and frequencies inner; the next
    // point's inputs are loaded (streaming: each is read once per hemisphere) before
    // the current one is solved
    int zz = 0, f = tid;
    bool live = f < nf;
    float xh = 0.0f, eh = 0.0f, be = 0.0f, nb = 0.0f, Jv = 0.0f, Pv = 0.0f;
    if (live) {
      const int c = dir > 0 ? k0 + i0 : k1 - 1 - i0;
      colf_load(A, f + nfs * c, xh, eh, be, nb, Jv, Pv);
    }
    while (live) {
      int zn = zz, fn = f + BS;
      if (fn >= nf) {
        zn = zz + 1;
        fn = tid;
      }
      const bool nlive = zn < zc;
      float xh2 = 0.0f, eh2 = 0.0f, be2 = 0.0f, nb2 = 0.0f, Jv2 = 0.0f, Pv2 = 0.0f;
      if (nlive) {
        const int cn = dir > 0 ? k0 + i0 + zn : k1 - 1 - (i0 + zn);
        colf_load(A, fn + nfs * cn, xh2, eh2, be2, nb2, Jv2, Pv2);
      }
      {
        const int c = dir > 0 ? k0 + i0 + zz : k1 - 1 - (i0 + zz);
        const float vz = sVz[zz], idf = sIdf[zz];
        const float *Cz = sC + (size_t)zz * nl * kColFusedConsts;
        const size_t o = f + nfs * c;
        const int p0 = sLp[f], n = sLp[f + 1] - p0;
        for (int d = 0; d < ND; d++) {
          const float muf = sDir[3 * d], dsup05 = sDir[3 * d + 1], w2 = sDir[3 * d + 2];
          ColfPoint P;
          colf_opacity(A, Cz, sLi, sLx, sq, f, p0, n, vz * muf, idf, xh, eh, be, P);
          // long_char_linear's step (k_long_char_columns)
          const float xx = P.chi, ss = P.S;
          const size_t u = (size_t)d * nf + f;
          const float xxup = sXu[u], ssup = sSu[u], Inuup = sIu[u];
          float dt = dsup05 * (xxup + xx);
          dt = fmaxf(dt, dtmax);
          float E, Wt, Psi, Esc;
          linear_weights(dt, E, Wt, Psi, Esc);
          float Inu = fma_t(Psi, ss, fma_t(Wt, ssup, Inuup * E));
          const bool off = dt <= 0 || xx <= 0 || fabsf(Inu) > Imax;
          const float Irem = fma_t(Wt, ssup, Inuup * E);
          Inu = fmaxf(-Imax, fminf(Imax, Inu));
          Psi = off ? 0.0f : Psi;
          const float irem = off ? Inu : Irem;
          const float esc = off ? 1.0f : Esc;
          const float ps = (dt > 0 && xx > 0) ? Psi / xx : 0.0f;
          Jv = fmaf(w2, Inu, Jv);
          Pv = fmaf(w2, ps, Pv);
          sXu[u] = xx;
          sSu[u] = ss;
          sIu[u] = Inu;
          // bound_bound_rates' terms of this point (k_bb_rates, split rates)
          float *T0 = sT + (size_t)d * 3 * ZR + (size_t)zz * RS, *T1 = T0 + ZR, *T3 = T1 + ZR;
          const float *wm = swm + (size_t)d * NS;
#pragma unroll
          for (int k = 0; k < kColFusedMaxLines; k++) {
            if (k < n) {
              const int i = sLx[p0 + k];
              const int *Li = sLi + kColFusedLineInts * i;
              const float *C = Cz + kColFusedConsts * i;
              const int slot = Li[0] + f - Li[1];
              const float phi = P.phi[k];
              const float vvv = phi * wm[slot];
              float t0, t1;
              if (A.precond) {
                float psi = ps;
                const float eta_u = phi * C[5];
                const float eta_t = eta_u * be;
                const float chi_t = phi * C[6] - eta_t;
                const float eta_other = be * other_contribution(eta_u, Li[2], P.oL, P.oR, P.oid);
                const float chi_other = other_contribution(phi * C[6], Li[2], P.cL, P.cR, P.cid) - eta_other;
                const float other = eta_other;
                if (chi_t < 0.0f) psi = 0.0f;
                const float up = psi == 0.0f ? Inu : irem + psi * other;
                const float spont = psi == 0.0f ? 1.0f : (chi_other + esc * chi_t) / xx;
                t0 = vvv * spont * (nb * C[7]);
                t1 = vvv * (up - nb * spont);
              } else {
                t0 = vvv * (nb * C[7]);
                t1 = vvv * (Inu - nb);
              }
              T0[slot] = t0;
              T1[slot] = t1;
              T3[slot] = phi * swq[slot];
            }
          }
        }
        __stcs(A.J + o, Jv);
        __stcs(A.PsiJ + o, Pv);
      }
      zz = zn;
      f = fn;
      live = nlive;
      xh = xh2;
      eh = eh2;
      be = be2;
      nb = nb2;
      Jv = Jv2;
      Pv = Pv2;
    }
    __syncthreads();
    // each (line, cell): for each direction in turn, the sums over the line's points
    // in ascending f, then the rates' update (the directions' order of k_bb_rates)
    for (int p = tid; p < nl * zc; p += BS) {
      const int i = p / zc, zz = p - i * zc;
      const int *Li = sLi + kColFusedLineInts * i;
      if (!Li[3]) continue;
      const int c = dir > 0 ? k0 + i0 + zz : k1 - 1 - (i0 + zz);
      const size_t kk = (size_t)c + (size_t)A.ncell * i;
      float gij = A.gw_ij[kk], gji = A.gw_ji[kk];
      for (int d = 0; d < ND; d++) {
        const float *r0 = sT + (size_t)d * 3 * ZR + (size_t)zz * RS + Li[0], *r1 = r0 + ZR, *r3 = r1 + ZR;
        float s0 = 0.0f, s1 = 0.0f, s3 = 0.0f;
        for (int k = 0; k < Li[4]; k++) {
          s0 = s0 + r0[k];
          s1 = s1 + r1[k];
          s3 = s3 + r3[k];
        }
        float g_th = s0, g_dev = s1;
        if (Li[3] == 2 && s3 > 0.0f) {
          g_th = g_th / (s3 * A.wtot);
          g_dev = g_dev / (s3 * A.wtot);
        }
        gij = gij + g_th;
        gji = gji + g_dev;
      }
      A.gw_ij[kk] = gij;
      A.gw_ji[kk] = gji;
    }
  }
}

}  // namespace m3d

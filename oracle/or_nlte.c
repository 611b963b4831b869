/*
 * or_nlte.c -- CPU restatement of the model-atom opacities and the ALI rate
 * integrals of OpenMULTI3D (non-hydrogen lines).  TEST INFRASTRUCTURE ONLY.
 *
 *   bound_bound_damping / line_damping   SRC/rt_patch_mod.f90:2649-2681, HOP/bbtrans_mod.f90:78-106
 *   add_bound_free_opacities             SRC/rt_patch_mod.f90:2581-2643
 *   foreground split start               SRC/rt_patch_mod.f90:1474-1487
 *   add_bound_bound_opacities            SRC/rt_patch_mod.f90:2689-2831
 *   add_largest / other_contribution     SRC/rt_patch_mod.f90:3150-3187
 *   work_to_transfer_units (split)       SRC/rt_patch_mod.f90:3571-3651
 *   bound_bound_rates                    SRC/rt_patch_mod.f90:2852-3142
 *   bound_free_rates                     SRC/rt_patch_mod.f90:3193-3259
 *   normalize_profiles                   SRC/atom_mod.f90:377-430
 *
 * real(4) locals assigned from real(8) expressions are rounded where the
 * Fortran assigns them; every sum runs in the reference's loop order.
 */
#include <float.h>
#include <math.h>
#include <stddef.h>

#include "m3d_oracle.h"
#include "or_nlte.h"

static inline float profile(const float *tgx, const float *th2x, float a, float q, float vpr, float idf)
{
  float h;
  or_qlg_bot_profile(tgx, th2x, 1, &a, &q, &vpr, &idf, &h);
  return h;
}

static inline int lact(const nl_window_t *w, int i) { return !w->lactive || w->lactive[i]; }
static inline int cact(const nl_window_t *w, int i) { return !w->cactive || w->cactive[i]; }

void or_bb_damping(const nl_window_t *w, int ncell, const float *ne, const float *tothi, const float *vbar2,
                   const float *stark_pe, const float *unsold, const float *inv_df, float *adamp)
{
  for (int i = 0; i < w->nline; i++) {
    if (!lact(w, i)) continue;
    for (int c = 0; c < ncell; c++) {
      /* the constants are real(8): each statement is evaluated in double and
       * stored to the real(4) adamp */
      float a = 0.0f;
      if (w->unsold[i]) a = (float)((double)a + w->gw1[i] * (double)unsold[c]);
      else a = (float)((double)a + (w->gw1[i] == 0.0 ? 0.0 : w->gw1[i] * pow((double)vbar2[c], w->gw2[i]) * (double)tothi[c]));
      if (w->gstk[i] >= 0.0) a = (float)((double)a + w->gstk[i] * (double)ne[c]);
      else a = (float)((double)a - w->gstk[i] * (double)stark_pe[c]);
      a = (float)((double)a + w->grad[i]);
      adamp[(size_t)c + (size_t)ncell * i] = a * inv_df[c];
    }
  }
}

void or_bf_opacity(const nl_window_t *w, int ncell, const double *b, const double *nstar, const double *pop_ratio,
                   const double *e_kT, float *xhat, float *ehat)
{
  const size_t nf = (size_t)w->nf;
  for (int i = 0; i < w->ncont; i++) {
    if (!cact(w, i)) continue;
    const int li = w->ci[i], lj = w->cj[i];
    const double dev = w->ev[lj] - w->ev[li];
    for (int c = 0; c < ncell; c++) {
      float ni, tmp;
      if (b) {
        ni = (float)(nstar[(size_t)c + (size_t)ncell * li] * b[(size_t)c + (size_t)ncell * li] * pop_ratio[c]);
        tmp = (float)(nstar[(size_t)c + (size_t)ncell * li] * b[(size_t)c + (size_t)ncell * lj] * pop_ratio[c]);
        if (dev * e_kT[c] > w->cut_x) tmp = 0.0f;
      } else {
        ni = (float)(nstar[(size_t)c + (size_t)ncell * li] * pop_ratio[c]);
        tmp = ni;
      }
      for (int f = w->cblue[i]; f <= w->cred[i]; f++) {
        const float alpha = w->alpha[w->coff[i] + f - w->cblue[i]];
        xhat[(size_t)f + nf * c] = xhat[(size_t)f + nf * c] + alpha * ni;
        ehat[(size_t)f + nf * c] = ehat[(size_t)f + nf * c] + alpha * tmp;
      }
    }
  }
}

static inline void add_largest(float value, int index, float *largest, float *rest, int *largest_index)
{
  if (fabsf(value) > fabsf(*largest)) {
    *rest = *rest + *largest;
    *largest = value;
    *largest_index = index;
  } else {
    *rest = *rest + value;
  }
}

static inline float other_contribution(float value, int index, float largest, float rest, int largest_index)
{
  return index == largest_index ? rest : largest + (rest - value);
}

void or_bb_opacity(const nl_window_t *w, int ncell, const double *b, const double *nstar, const double *pop_ratio,
                   const double *e_kT, const float *inv_df, const float *vproj, const float *adamp,
                   const float *tgx, const float *th2x, int lte, int split, float wmu, float *xhat, float *ehat,
                   float *sopL, float *sopR, int *sid, float *schL, float *schR, int *schid, float *wphi)
{
  const size_t nf = (size_t)w->nf;
  if (split)
    for (size_t k = 0; k < nf * ncell; k++) {
      sopL[k] = ehat[k];
      sopR[k] = 0.0f;
      sid[k] = 0;
      schL[k] = xhat[k];
      schR[k] = 0.0f;
      schid[k] = 0;
    }
  float vphi[4096];
  for (int i = 0; i < w->nline; i++) {
    if (!lact(w, i)) continue;
    const int li = w->li[i], lj = w->lj[i], fs = w->lblue[i], fe = w->lred[i], off = w->loff[i];
    const float lower_off = (float)(w->lower_ev[i] - w->ev[li]);
    for (int c = 0; c < ncell; c++) {
      const float idf = inv_df[c], ekt = (float)e_kT[c];
      const float ni = (float)(nstar[(size_t)c + (size_t)ncell * li] * pop_ratio[c]);
      float bi = 1.0f, bj = 1.0f;
      if (!lte && b) {
        bi = (float)b[(size_t)c + (size_t)ncell * li];
        bj = (float)b[(size_t)c + (size_t)ncell * lj];
      }
      if (lower_off != 0.0f) {
        bi = bi * expf(-lower_off * ekt);
        bj = bj * expf(-lower_off * ekt);
      }
      const float vpr = vproj[c], a = adamp[(size_t)c + (size_t)ncell * i];
      for (int f = fs; f <= fe; f++) vphi[f - fs] = profile(tgx, th2x, a, w->q[off + f - fs], vpr, idf);
      const float Rij = (float)((double)ni * w->Bij[i]);
      const float eta_fac = Rij * bj, chi_fac = Rij * bi;
      for (int f = fs; f <= fe; f++) {
        const size_t k = (size_t)f + nf * c;
        xhat[k] = xhat[k] + vphi[f - fs] * chi_fac;
        ehat[k] = ehat[k] + vphi[f - fs] * eta_fac;
      }
      if (split)
        for (int f = fs; f <= fe; f++) {
          const size_t k = (size_t)f + nf * c;
          add_largest(vphi[f - fs] * eta_fac, w->lindex[i], &sopL[k], &sopR[k], &sid[k]);
          add_largest(vphi[f - fs] * chi_fac, w->lindex[i], &schL[k], &schR[k], &schid[k]);
        }
      if (wphi && w->lsums[i]) {
        /* sum(phi * line%wq): real(8) products summed in real(8), stored to real(4) */
        double s = 0.0;
        for (int f = fs; f <= fe; f++) s = s + (double)vphi[f - fs] * w->wq[off + f - fs];
        const size_t kw = (size_t)c + (size_t)ncell * w->lntrans[i];
        wphi[kw] = wphi[kw] + wmu * (float)s;
      }
    }
  }
}

int or_transfer_units_split(int nf, int ncell, float *w1, float *w2, const float *beta, const float *sopL,
                            const float *sopR, const float *scat, double maser_chi_floor, int suppress_masers)
{
  int nfl = 0;
  const float fl = (float)maser_chi_floor;
  for (size_t k = 0; k < (size_t)nf * ncell; k++) {
    const float eta_rest = beta[k] * sopR[k];
    float eta = beta[k] * sopL[k] + eta_rest;
    float chi = w1[k] - eta;
    if (scat) eta = beta[k] * sopL[k] + (eta_rest + scat[k]);
    const float xhat = w1[k];
    const float floor_ = fmaxf(fl * fabsf(xhat), FLT_MIN);
    if (suppress_masers) chi = fmaxf(chi, floor_);
    else if (fabsf(chi) < floor_) {
      chi = copysignf(floor_, chi);
      nfl++;
    }
    w1[k] = chi;
    w2[k] = eta / chi;
  }
  return nfl;
}

void or_bb_rates(const nl_window_t *w, const nl_rate_opts_t *o, int ncell, const double *b, const double *nstar,
                 const double *pop_ratio, const double *e_kT, const float *inv_df, const float *vproj,
                 const float *adamp, const float *tgx, const float *th2x, const float *work1, const float *inu,
                 const float *psi_a, const float *irem, const float *escape, const float *beta, const float *Bnu,
                 const float *sopL, const float *sopR, const int *sid, const float *schL, const float *schR,
                 const int *schid, const float *scat, const unsigned *flags_in, unsigned *flags_raise, int nwords,
                 float *gamma_ij, float *gamma_ji)
{
  const size_t nf = (size_t)w->nf;
  float vph[4096], wmunu[4096], wqf[4096];
  for (int i = 0; i < w->nline; i++) {
    if (!lact(w, i)) continue;
    const int li = w->li[i], lj = w->lj[i], fs = w->lblue[i], fe = w->lred[i], off = w->loff[i];
    for (int f = fs; f <= fe; f++) {
      wmunu[f - fs] = (float)((double)o->wmu * w->wnu[off + f - fs] * w->Aij[i]);
      wqf[f - fs] = (float)w->wq[off + f - fs];
    }
    const int own_norm = o->per_direction && !w->lsums[i];
    const float lower_off = (float)(w->lower_ev[i] - w->ev[li]);
    const int index = w->lindex[i];
    for (int c = 0; c < ncell; c++) {
      const double nsi = nstar[(size_t)c + (size_t)ncell * li], nsj = nstar[(size_t)c + (size_t)ncell * lj];
      const double bbi = b[(size_t)c + (size_t)ncell * li], bbj = b[(size_t)c + (size_t)ncell * lj];
      float ni = (float)(bbi * nsi), nj = (float)(bbj * nsj);
      const float idf = inv_df[c], vpr = vproj[c], a = adamp[(size_t)c + (size_t)ncell * i];
      const float ekt = (float)e_kT[c];
      float inv_nref = 0.0f;
      if (nsi > 0 && nsj > 0) {
        const double beta_ref = nsj * w->g[li] / (nsi * w->g[lj]);
        inv_nref = (float)fmin((1.0 - beta_ref) / beta_ref, 1e35);
      }
      if (lower_off != 0.0f) {
        ni = ni * expf(-lower_off * ekt);
        nj = nj * expf(-lower_off * ekt);
      }
      float eta_coef = 0.0f, abs_coef = 0.0f, g_ratio = 0.0f;
      if (o->precond) {
        float split_bj = (float)bbj;
        if (lower_off != 0.0f) split_bj = split_bj * expf(-lower_off * ekt);
        float split_Rij = (float)(nsi * pop_ratio[c]);
        split_Rij = (float)((double)split_Rij * w->Bij[i]);
        eta_coef = split_Rij * split_bj;
        float split_bi = (float)bbi;
        if (lower_off != 0.0f) split_bi = split_bi * expf(-lower_off * ekt);
        abs_coef = split_Rij * split_bi;
        g_ratio = 0.0f;
        if (nj > 0.0f) g_ratio = (float)((double)(ni / nj) * (w->g[lj] / w->g[li]));
      }
      float sum_A = 0, sum_I = 0, sum_P = 0, sum_T = 0, sum_U = 0, sum_w = 0;
      if (o->split) {
        for (int f = fs; f <= fe; f++) vph[f - fs] = profile(tgx, th2x, a, w->q[off + f - fs], vpr, idf);
      } else {
        for (int f = fs; f <= fe; f++) {
          const size_t k = (size_t)f + nf * c;
          const float phi = profile(tgx, th2x, a, w->q[off + f - fs], vpr, idf);
          const float vvv = phi * wmunu[f - fs];
          if (own_norm) sum_w = sum_w + phi * wqf[f - fs];
          sum_A = sum_A + vvv * (Bnu[k] * inv_nref);
          sum_I = sum_I + vvv * inu[k];
          sum_P = sum_P + vvv * phi * psi_a[k] * beta[k];
        }
      }
      if (o->split && o->precond) {
        const int t = w->lntrans[i], pw = t / 32, pb = t % 32;
        int in_force = 0, raise = 0;
        if (o->use_flags) in_force = (flags_in[(size_t)c + (size_t)ncell * pw] >> pb) & 1u;
        for (int f = fs; f <= fe; f++) {
          const size_t k = (size_t)f + nf * c;
          const float v = vph[f - fs];
          float psi = psi_a[k];
          const float eta_u = v * eta_coef;
          const float eta_t = eta_u * beta[k];
          const float chi_t = v * abs_coef - eta_t;
          const float eta_other = beta[k] * other_contribution(eta_u, index, sopL[k], sopR[k], sid[k]);
          const float chi_other = other_contribution(v * abs_coef, index, schL[k], schR[k], schid[k]) - eta_other;
          float other = eta_other;
          if (o->do_scat) other = other + scat[k];
          if (chi_t < 0.0f || in_force) psi = 0.0f;
          raise = raise || psi == 0.0f;
          const float up = psi == 0.0f ? inu[k] : irem[k] + psi * other;
          const float spont = psi == 0.0f ? 1.0f : (chi_other + escape[k] * chi_t) / work1[k];
          const float vvv = v * wmunu[f - fs];
          const float nb = Bnu[k];
          sum_T = sum_T + vvv * spont * (nb * inv_nref);
          sum_U = sum_U + vvv * (up - nb * spont);
        }
        if (o->use_flags && raise && !in_force) flags_raise[(size_t)c + (size_t)ncell * pw] |= 1u << pb;
      } else if (o->split) {
        for (int f = fs; f <= fe; f++) {
          const size_t k = (size_t)f + nf * c;
          const float vvv = vph[f - fs] * wmunu[f - fs];
          const float nb = Bnu[k];
          sum_T = sum_T + vvv * (nb * inv_nref);
          sum_U = sum_U + vvv * (inu[k] - nb);
        }
      }
      float g_th, g_dev;
      if (o->split) {
        g_th = sum_T;
        g_dev = sum_U;
      } else {
        g_th = sum_A;
        g_dev = sum_I;
        if (o->precond) {
          g_th = g_th - sum_P * eta_coef * (g_ratio - 1.0f);
          g_dev = g_dev - sum_P * eta_coef;
        }
        if (inv_nref > 0.0f) g_dev = g_dev - g_th / inv_nref;
      }
      if (own_norm) {
        if (o->split) {
          sum_w = 0.0f;
          for (int f = fs; f <= fe; f++) sum_w = sum_w + vph[f - fs] * wqf[f - fs];
        }
        if (sum_w > 0.0f) {
          g_th = g_th / (sum_w * o->wtot);
          g_dev = g_dev / (sum_w * o->wtot);
        }
      }
      gamma_ij[(size_t)c + (size_t)ncell * i] = gamma_ij[(size_t)c + (size_t)ncell * i] + g_th;
      gamma_ji[(size_t)c + (size_t)ncell * i] = gamma_ji[(size_t)c + (size_t)ncell * i] + g_dev;
    }
  }
  (void)nwords;
}

void or_bf_rates(const nl_window_t *w, int ncell, int precond, const double *b, const double *nstar,
                 const double *e_kT, const float *twohnu3_c2, const float *Jnu, const float *PsiJ, const float *beta,
                 float *gamma_ij, float *gamma_ji)
{
  const size_t nf = (size_t)w->nf;
  float wal[4096];
  for (int j = 0; j < w->ncont; j++) {
    if (!cact(w, j)) continue;
    const int i = j + w->nline, li = w->ci[j], lj = w->cj[j], fs = w->cblue[j], fe = w->cred[j], off = w->coff[j];
    for (int f = fs; f <= fe; f++) {
      const float wmunu = (float)(0.5 * w->cwnu[off + f - fs]);
      wal[f - fs] = twohnu3_c2[f] * w->alpha[off + f - fs] * wmunu;
    }
    const double dev = w->ev[lj] - w->ev[li];
    for (int c = 0; c < ncell; c++) {
      if (dev * e_kT[c] > w->cut_x) continue;
      float sum_abs = 0, sum_ems = 0, sum_pre = 0;
      for (int f = fs; f <= fe; f++) {
        const size_t k = (size_t)f + nf * c;
        const float vij = wal[f - fs];
        const float vji = vij * beta[k];
        const float phi = PsiJ[k] * w->alpha[off + f - fs];
        sum_abs = sum_abs + vij * Jnu[k];
        sum_ems = sum_ems + vji * (Jnu[k] + 1.0f);
        sum_pre = sum_pre + vji * phi;
      }
      float g_ij = sum_abs, g_ji = sum_ems;
      if (precond) {
        const double nsi = nstar[(size_t)c + (size_t)ncell * li];
        g_ij = (float)((double)g_ij - (double)sum_pre * nsi * b[(size_t)c + (size_t)ncell * lj]);
        g_ji = (float)((double)g_ji - (double)sum_pre * nsi * b[(size_t)c + (size_t)ncell * li]);
      }
      gamma_ij[(size_t)c + (size_t)ncell * i] = gamma_ij[(size_t)c + (size_t)ncell * i] + g_ij;
      gamma_ji[(size_t)c + (size_t)ncell * i] = gamma_ji[(size_t)c + (size_t)ncell * i] + g_ji;
    }
  }
}

void or_normalize_profiles(int ncell, int nline, int nrad, const int *ti, const int *tj,
                           const unsigned char *active, const unsigned char *has_wphi, int first_iter,
                           const double *nstar, float *wphi, float *gamma_ij, float *gamma_ji)
{
  if (first_iter)
    for (int i = 0; i < nline; i++) {
      if ((active && !active[i]) || !has_wphi[i]) continue;
      for (int c = 0; c < ncell; c++) {
        float *v = &wphi[(size_t)c + (size_t)ncell * i];
        *v = *v > 0.0f ? 1.0f / *v : 1.0f;
      }
    }
  for (int i = 0; i < nline; i++) {
    if ((active && !active[i]) || !has_wphi[i]) continue;
    for (int c = 0; c < ncell; c++) {
      const size_t k = (size_t)c + (size_t)ncell * i;
      gamma_ij[k] = gamma_ij[k] * wphi[k];
      gamma_ji[k] = gamma_ji[k] * wphi[k];
    }
  }
  for (int i = nline; i < nrad; i++) {
    if (active && !active[i]) continue;
    for (int c = 0; c < ncell; c++) {
      const size_t k = (size_t)c + (size_t)ncell * i;
      gamma_ji[k] = (float)((double)gamma_ji[k] *
                            (nstar[(size_t)c + (size_t)ncell * ti[i]] / nstar[(size_t)c + (size_t)ncell * tj[i]]));
    }
  }
}

/* lte_background_emission (rt_patch_mod.f90:2127-2328) with convert_to_work_units
 * (:3518-3536); jmode 0: Jnu given, 1: Jnu = Bnu, 2: Jnu = 0; PsiJ non-NULL: the OAB
 * step (:2225-2252); returns the number of negative OAB results */
long long or_lte_emission(size_t n, const float *chi, const float *sigma, const float *Bnu, const float *beta,
                          const float *J, int jmode, const float *PsiJ, float *Jali, int jali_valid, double op_max,
                          float *xhat, float *ehat, float *dJnu)
{
  long long neg = 0;
  for (size_t k = 0; k < n; k++) {
    const float B = Bnu[k];
    float j = jmode == 1 ? B : (jmode == 2 ? 0.0f : J[k]);
    if (jmode == 0 && PsiJ) {
      double op = (double)(sigma ? sigma[k] : 0.0f) * (double)PsiJ[k];
      op = fmax(0.0, fmin(op, op_max));
      const double jfs = (double)j;
      const double jold = jali_valid ? (double)Jali[k] : jfs;
      double jn = (jfs - op * jold) / (1.0 - op);
      if (jn < 0.0) {
        jn = jfs;
        neg++;
      }
      j = (float)jn;
      Jali[k] = j;
    }
    const float dj = j - B;
    const float eta = chi[k] * B + (sigma ? sigma[k] : 0.0f) * dj;
    if (dJnu) dJnu[k] = dj;
    xhat[k] = chi[k] + eta;
    ehat[k] = eta / beta[k];
  }
  return neg;
}

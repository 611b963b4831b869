/*
 * or_nlte.h -- CPU restatement of OpenMULTI3D's model-atom opacities and ALI
 * rate integrals (non-hydrogen lines).  TEST INFRASTRUCTURE ONLY: the checker
 * of the NLTE kernels, never the product.
 *
 * Layouts: (f, cell) arrays frequency fastest; (cell, k) arrays cell fastest;
 * 0-based indices.  A line's points f = blue..red of the window sit at
 * q[off + f - blue] (likewise wnu, wq); a continuum's at alpha[off + f - blue].
 */
#ifndef OR_NLTE_H
#define OR_NLTE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nl_window {
  int nf, nline, ncont, nlevel;
  /* lines */
  const int *li, *lj;            /* levels */
  const int *lntrans;            /* transition index in the atom (gamma, wphi, psi_flags) */
  const int *lindex;             /* split-tracking contribution index (>= 1) */
  const int *lblue, *lred, *loff;
  const float *q;                /* per line point, real(4) */
  const double *wnu, *wq;        /* per line point, real(8) */
  const double *Bij, *Aij, *lower_ev;   /* real(8) line constants (bbtrans_mod.f90:20-21) */
  const unsigned char *lactive;  /* or NULL */
  const unsigned char *lsums;    /* sums_over_windows */
  const double *grad, *gw1, *gw2, *gstk;
  const unsigned char *unsold;
  /* continua */
  const int *ci, *cj, *cntrans, *cblue, *cred, *coff;
  const float *alpha;            /* per continuum point, real(4) */
  const double *cwnu;            /* per continuum point, real(8) */
  const unsigned char *cactive;  /* or NULL */
  /* levels */
  const double *g, *ev;
  double cut_x;
} nl_window_t;

/* bound_bound_damping (rt_patch_mod.f90:2649-2681), line_damping (bbtrans_mod.f90:78-106):
 * adamp(cell, line) = damping x inv_df */
void or_bb_damping(const nl_window_t *w, int ncell, const float *ne, const float *tothi, const float *vbar2,
                   const float *stark_pe, const float *unsold, const float *inv_df, float *adamp);

/* add_bound_free_opacities (rt_patch_mod.f90:2581-2643): xhat, ehat (nf, ncell) */
void or_bf_opacity(const nl_window_t *w, int ncell, const double *b, const double *nstar, const double *pop_ratio,
                   const double *e_kT, float *xhat, float *ehat);

/* the split-tracking start of foreground (rt_patch_mod.f90:1474-1487) plus
 * add_bound_bound_opacities (:2689-2831) for one direction */
void or_bb_opacity(const nl_window_t *w, int ncell, const double *b, const double *nstar, const double *pop_ratio,
                   const double *e_kT, const float *inv_df, const float *vproj, const float *adamp,
                   const float *tgx, const float *th2x, int lte, int split, float wmu, float *xhat, float *ehat,
                   float *sopL, float *sopR, int *sid, float *schL, float *schR, int *schid, float *wphi);

/* work_to_transfer_units with split rates (rt_patch_mod.f90:3571-3651); scat
 * = chi_scat*dJnu or NULL; returns the number of floored points */
int or_transfer_units_split(int nf, int ncell, float *w1, float *w2, const float *beta, const float *sopL,
                            const float *sopR, const float *scat, double maser_chi_floor, int suppress_masers);

/* bound_bound_rates for one direction (rt_patch_mod.f90:2852-3142);
 * gamma_ij/ji are the window's (ncell, nline + ncont) */
typedef struct nl_rate_opts {
  int split, precond, per_direction, use_flags, do_scat, pad;
  float wmu, wtot;
} nl_rate_opts_t;

void or_bb_rates(const nl_window_t *w, const nl_rate_opts_t *o, int ncell, const double *b, const double *nstar,
                 const double *pop_ratio, const double *e_kT, const float *inv_df, const float *vproj,
                 const float *adamp, const float *tgx, const float *th2x, const float *work1, const float *inu,
                 const float *psi, const float *irem, const float *escape, const float *beta, const float *Bnu,
                 const float *sopL, const float *sopR, const int *sid, const float *schL, const float *schR,
                 const int *schid, const float *scat, const unsigned *flags_in, unsigned *flags_raise, int nwords,
                 float *gamma_ij, float *gamma_ji);

/* bound_free_rates (rt_patch_mod.f90:3193-3259) */
void or_bf_rates(const nl_window_t *w, int ncell, int precond, const double *b, const double *nstar,
                 const double *e_kT, const float *twohnu3_c2, const float *Jnu, const float *PsiJ, const float *beta,
                 float *gamma_ij, float *gamma_ji);

/* normalize_profiles (atom_mod.f90:377-430) on the atom's (ncell, nrad) rates;
 * wphi (ncell, nline_atom) with has_wphi (nline_atom) */
void or_normalize_profiles(int ncell, int nline, int nrad, const int *ti, const int *tj,
                           const unsigned char *active, const unsigned char *has_wphi, int first_iter,
                           const double *nstar, float *wphi, float *gamma_ij, float *gamma_ji);

/* lte_background_emission with convert_to_work_units (rt_patch_mod.f90:2127-2328, 3518-3536) */
long long or_lte_emission(size_t n, const float *chi, const float *sigma, const float *Bnu, const float *beta,
                          const float *J, int jmode, const float *PsiJ, float *Jali, int jali_valid, double op_max,
                          float *xhat, float *ehat, float *dJnu);

#ifdef __cplusplus
}
#endif
#endif

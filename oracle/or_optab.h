/*
 * or_optab.h -- CPU restatement of OpenMULTI3D's sampled opacity tables
 * (HOP/optab_mod.f90).  TEST INFRASTRUCTURE ONLY: the checker of the table
 * kernels, never the product.
 *
 * A table component is (nnu, ntemp, nne) fp32 with the wavelength fastest, over
 * the fp64 wavelength nodes lam and two regular PC axes of (ln T, ln ne).
 * Cell fields are flat (ncell); (f, cell) arrays have the frequency fastest.
 */
#ifndef OR_OPTAB_H
#define OR_OPTAB_H

#ifdef __cplusplus
extern "C" {
#endif

/* pca_transform_type (optab_mod.f90:26-31); rot in Fortran order rot(1,1), rot(2,1), rot(1,2), rot(2,2) */
typedef struct or_pca {
  double mu[2], rot[4], c0[2], dc[2];
} or_pca_t;

/* sample_build_derivatives (optab_mod.f90:125-166) for one component: dl along
 * the wavelength on the fp64 nodes, dt and de along the PC axes. */
void or_optab_slopes(int nnu, int ntemp, int nne, const double *lam, const float *val, const or_pca_t *pca,
                     float *dl, float *dt, float *de);

/* sample_interpolate (optab_mod.f90:181-287): back = (kappa + kappa_scat) chi500,
 * scat = kappa_scat chi500, (nf, ncell). */
int or_optab_sample(int nnu, int ntemp, int nne, const double *lam, const or_pca_t *pca, const float *val,
                    const float *dl, const float *dt, const float *de, const float *sv, const float *sl,
                    const float *st, const float *se, long long ncell, const double *temp, const double *ne,
                    const float *chi500, int nf, const double *lam_q, float *back, float *scat);

/* sample_interpolate_ll (optab_mod.f90:300-409): per cell the query wavelength
 * lam_q (1 + vproj); xhat and ehat (nf, ncell) += kappa chi500, and with the
 * scattering component given chi_scat += kappa_scat chi500. */
int or_optab_sample_ll(int nnu, int ntemp, int nne, const double *lam, const or_pca_t *pca, const float *val,
                       const float *dl, const float *dt, const float *de, const float *sv, const float *sl,
                       const float *st, const float *se, long long ncell, const double *temp, const double *ne,
                       const float *chi500, const float *vproj, int nf, const double *lam_q, float *xhat,
                       float *ehat, float *chi_scat);

#ifdef __cplusplus
}
#endif
#endif

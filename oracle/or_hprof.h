/*
 * or_hprof.h -- CPU restatement of OpenMULTI3D's hydrogen line profiles
 * (HOP/hprofl_mod.f90, the analytic path).  TEST INFRASTRUCTURE ONLY: the checker
 * of the hydrogen kernels, never the product.
 *
 * Per-cell arrays are flat (ncell); chi, eta and cont are (nf, ncell), frequency
 * fastest; frequency indices are 0-based.
 */
#ifndef OR_HPROF_H
#define OR_HPROF_H

#ifdef __cplusplus
extern "C" {
#endif

/* hline_t (hprofl_mod.f90:156-165) */
typedef struct or_hline {
  int n, m, bpo, io;
  int opts, pad;             /* the switches it was built with (disable_vdw reaches hcell_prepare) */
  double nu0, grad, gstk, gw1, gw2, gw3;
  double dq[14], wt[14];
  double dqbar, dqmax, qray;
} or_hline_t;

/* the per-cell inputs of add_h_opacities (hprofl_mod.f90:208-234) */
typedef struct or_hcells {
  const float *vproj, *inv_df, *temp, *ni, *ne, *tothi, *vbar2h, *fo, *t3nhe;
} or_hcells_t;

/* switches of bbtrans_mod / hprofl_mod: disable_rad 1, disable_stk 2, disable_vdw 4, no hydrogen_BPO 8 */
void or_hydrogen_line(int n, int m, double nu0, unsigned opts, or_hline_t *h);

/* hcell_prepare + hprofile for one cell at the detunings q (n points); phi out */
void or_hprofile(const or_hline_t *h, const float *tgx, const float *th2x, float temp, float ne, float fo,
                 float vbar2h, float tothi, float t3nhe, float idf, int n, const double *q, float *phi);

/* add_h_opacities (hprofl_mod.f90:208-385), analytic profiles: chi, eta (nf, ncell)
 * += the line; bi, bj NULL for LTE.  line_used, line_strength raised. */
void or_add_h_opacities(const or_hline_t *h, const float *tgx, const float *th2x, double Bij, int f0, int nf,
                        const double *nu, long long ncell, const or_hcells_t *cells, const float *bi,
                        const float *bj, float *chi, float *eta, const float *cont, int *line_used,
                        float *line_strength);

#ifdef __cplusplus
}
#endif
#endif

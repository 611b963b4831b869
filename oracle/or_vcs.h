/*
 * or_vcs.h -- the tabulated hydrogen profiles of HOP/hvcs_mod.f90, restated for
 * the oracle.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef OR_VCS_H
#define OR_VCS_H

#ifdef __cplusplus
extern "C" {
#endif

#define OR_VCS_NW 44   /* delta-lambda points */
#define OR_VCS_NT 4    /* temperature nodes */
#define OR_VCS_NE 13   /* electron-density nodes */
#define OR_VCS_NH 13   /* hydrogen-density nodes */
#define OR_VCS_NL 18   /* lines per series */

typedef struct {
  int loaded, nlines, radiative;
  int nlow[OR_VCS_NL], nup[OR_VCS_NL], nhhnr[OR_VCS_NL];
  float grid[OR_VCS_NL][OR_VCS_NE][OR_VCS_NT][OR_VCS_NH][OR_VCS_NW];   /* grid_vcs(i,j,kk,l,k) */
  float tslope[OR_VCS_NL][OR_VCS_NE][OR_VCS_NT][OR_VCS_NW];
  float nw[OR_VCS_NW], nt[OR_VCS_NT], ne[OR_VCS_NE], nh[OR_VCS_NH], dw_lin[OR_VCS_NW], nw_invdx;
  double dw_first, dw_last;
} or_vcs_series_t;

/* vcs_profile_t (hvcs_mod.f90:94-104) */
typedef struct {
  float lp[OR_VCS_NW];
  double lognorm, lam0, q_tail, ta, ts;
  int ok;
} or_vcs_cell_t;

int or_vcs_load(int series, const char *fname, int radiative);   /* 0 on success */
void or_vcs_clear(void);
const or_vcs_series_t *or_vcs_series(int series);
int or_vcs_row(int n, int m);
int or_vcs_supported(int n, int m);
int or_vcs_resonance(int n, int m);
int or_vcs_radiative(int n);
void or_vcs_prepare(int n, int m, double nu0, float temp, float ne, float nh, or_vcs_cell_t *c);
double or_vcs_eval(const or_vcs_cell_t *c, double q);
double or_vcs_tail(const or_vcs_cell_t *c, double lnq);

#ifdef __cplusplus
}
#endif
#endif

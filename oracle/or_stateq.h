/*
 * or_stateq.h -- CPU restatement of OpenMULTI3D's statistical-equilibrium step
 * (rate matrix, collisions, dense solves, population update, Ng extrapolation).
 * TEST INFRASTRUCTURE ONLY: the checker of the SE kernels, never the product.
 *
 * Level and transition indices are 0-based; per-cell arrays keep the cell
 * index fastest, a(cell, k) at a[cell + ncell*k], as the reference's
 * (x, y, z, level) arrays do.
 */
#ifndef OR_STATEQ_H
#define OR_STATEQ_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* collision pair kinds of classic_col (atom_mod.f90:1758-1880): electron recipes in
 * ckind, hydrogen recipes in chkind */
enum { SQ_COL_REGEMORTER = 1, SQ_COL_SEATON = 2 };
enum { SQ_COLH_DRAWIN = 1, SQ_COLH_TAKEDA = 2 };
/* gencol's record kinds (atom_mod.f90:2288-2344) */
enum { SQ_GC_NONE = 0, SQ_GC_OHM, SQ_GC_CE, SQ_GC_CH, SQ_GC_CHI, SQ_GC_CI, SQ_GC_CH0, SQ_GC_UP, SQ_GC_DN };

typedef struct sq_atom {
  int nlevel, nrad, nline;     /* transitions 0..nline-1 are lines, nline..nrad-1 continua */
  int ncol;                    /* collision pairs */
  const int *ti, *tj;          /* [nrad] lower / upper level */
  const unsigned char *active; /* [nrad] or NULL (all active) */
  const double *Aji;           /* [nrad] line Einstein A [1/s] (continua unused) */
  const double *g, *ev;        /* [nlevel] weight, energy above ground [eV] */
  const int *ion;              /* [nlevel] ion stage (1 = neutral) */
  const int *ci, *cj, *ckind;  /* [ncol] pair (i < j) and SQ_COL_* */
  const float *cfac;           /* [ncol] cdata of the pair (real(4)): f of a line, alpha0 of a continuum, 0 = none */
  double fmin, cbbesc, cbfesc, colscale, upsilon_floor; /* classic_col factors */
  double cut_x, bf_cut_rate;   /* radiative cut (atom_mod.f90:256-257) */
  const int *chkind;           /* [ncol] SQ_COLH_* or NULL: no hydrogen recipes */
  double drawin;               /* sq_prepare_drawin(awgt) */
  double cbbhsc, cbfhsc;       /* factors on the hydrogen rates */
  /* gencol's records (atom_mod.f90:2223-2360): ln of the rate coefficient on tgrid
   * and its node slopes, both (ngrec, ntemp) with the temperature fastest */
  int ngrec, ntemp, ch0_hmip, pad;
  const double *gt, *glnc, *gdc;
  const int *gll, *gul, *gkind, *gcoll; /* gcoll: collider row of UP/DN records, or NULL */
} sq_atom_t;

typedef struct sq_params {
  double max_update, sor_w, min_pop_frac, conv_pop_floor;
  double tmax_update; /* cells with temp >= tmax_update are left alone (needs temp) */
  double cswitch;     /* factor on the collision matrix; 0 leaves collisions out */
  int solver;         /* 0 lineq_no_pivot (== eqsyst), 1 lineq (full pivot), 2 LU partial pivot */
} sq_params_t;

typedef struct sq_result {
  double maxerr;        /* signed largest (weighted) relative change */
  long long epos_cell;  /* its cell, -1 if no change */
  int epos_level;       /* its level, -1 if no change */
  long long nclamp, ntot;
  long long nonfinite_cell; /* first cell whose solve was not finite (left unchanged), -1 if none */
} sq_result_t;

double sq_expin(double x);
double sq_gaunt(double lam, int n);
double sq_kramer(double lam, double dev);

/* prepare_Drawin's prefactor for an atom of weight awgt [amu] (atom_mod.f90:1741-1750) */
double sq_prepare_drawin(double awgt);

/* hermite_derivative (interpol_mod.f90:544-553): pchip_slopes8 over a whole line */
void sq_hermite_derivative(int n, const double *x, const double *y, double *d);
/* hermite_interpolation_single (interpol_mod.f90:558-578) */
double sq_hermite_interp(int n, const double *x, const double *y, const double *d, double xx);

/* cup (ncell, rows) of collision_rates (atom_mod.f90:918-930): ncol rows of the
 * electron rates, with chkind ncol more of the hydrogen rates, then with records
 * ngrec rows of their upward and ngrec of their downward rates.  nh1 (ncell) the
 * hydrogen ground-level density, nstar (ncell, nlevel), lsaha (ncell) and coll
 * (ncollider, ncell) are read where the recipes and records need them. */
void or_collisions(const sq_atom_t *at, int ncell, const double *temp, const double *ne, const double *e_kT,
                   const double *dxi, const double *nh1, const double *nstar, const double *lsaha,
                   const double *coll, double *cup);

void sq_lineq_no_pivot(double *a, double *b, int n);
void sq_lineq(double *a, double *b, int n);
void sq_lu_partial(double *a, double *b, int n);

void or_rate_matrix(const sq_atom_t *at, const sq_params_t *pr, const double *bl, const double *ns, double totn,
                    double e_kT, const float *gij, const float *gji, const double *cupc, double *w, double *e);

int or_stateq_update(const sq_atom_t *at, const sq_params_t *pr, int ncell, double *b, const double *nstar,
                     const double *totn, const double *temp, const double *e_kT, const float *gamma_ij,
                     const float *gamma_ji, const double *cup, sq_result_t *res, double *lvlerr);

void or_ng_accumulate(int ncell, int nlevel, const double *b, const double *oldb, double *gram);
int or_ng_extrapolate(int ncell, int nlevel, double *b, const double *oldb, const double *nstar, const double *totn,
                      double a, double bc, double max_change, double *emax, long long *epos_cell, int *epos_level);

#ifdef __cplusplus
}
#endif
#endif

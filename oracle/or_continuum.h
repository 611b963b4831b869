/*
 * or_continuum.h -- CPU restatement of HOP's continuum opacity of a window:
 * composition_type%continuum_opacities (HOP/composition_mod.f90:2893-2984) with
 * add_hrest (:3807-3846), electron_scattering (:3851-3872), rayleigh_scattering
 * (:3878-3939), boltzmann_factor (:2822-2852), and the absdat components of
 * bftrans_mod.f90 (load_lam_interp_weights :100-198, interp_xkap :235-452,
 * absorption_factor :476-531, add_absorption :537-594), with the 'H BF' levels
 * under occupation probabilities through wcalc2 and calc_x_and_k
 * (HOP/level_mod.f90:77-94, 149-279).  TEST INFRASTRUCTURE ONLY: the checker of
 * the continuum kernels, never the product.
 *
 * The EOS state (temperatures, electron pressure, the particles' number densities
 * and partition functions) and the components' tables are inputs.  Layouts: cell
 * arrays (ncell); window arrays (nlam, ncell), wavelength fastest; a table
 * xkap (nnu, ntt), wavelength fastest, as set_table stores it.  The structs have
 * the layout of m3d_bf_comp_t and m3d_cont_cells_t in include/m3dgpu.h.
 */
#ifndef OR_CONTINUUM_H
#define OR_CONTINUUM_H

#ifdef __cplusplus
extern "C" {
#endif

/* absorption_factor's cases (bftrans_mod.f90:500-528) */
enum {
  OR_BF_HMINUS = 1,   /* 'H- BF': n */
  OR_BF_NPE = 2,      /* 'H- FF', 'H2-', 'HE-': n Pe */
  OR_BF_H = 3,        /* 'H BF': 2.0898e-26/(2 k^5) n_k, or wcalc2 with occupation */
  OR_BF_H_FF = 4,     /* 'H FF' */
  OR_BF_PAIR = 5,     /* 'H+H', 'H+HE', 'H2+H', 'H2+H2', 'H2+HE': n n2 */
  OR_BF_H2PLUS = 6,   /* 'H2+': 1e-40 n n2 */
  OR_BF_PEDEP = 7,    /* Pe-dependent: n Pe */
  OR_BF_PEACH = 8,    /* Pe-dependent Peach table: 1e-40/e e_kT n Pe */
  OR_BF_MOLECULAR = 9,/* n awgt / N_A */
  OR_BF_REGULAR = 10  /* g exp(-xion e_kT - ln U) n */
};

typedef struct or_bf_comp {
  int kind, istim, nnu, ntt;
  int ilogl, kvadl, minex, maxex, loglam;
  int kvadt, minet, maxet, iteta, lam3, log_table;
  int k;
  const double *lam, *lnlam, *tt;
  const float *xkap;
  const unsigned char *ldisk;
  double xkap_scale, mint, maxt, minl, maxl;
  double ion_xion, level_g, level_xion, awgt;
  const double *n, *n2, *part, *level_n;
  /* 'H BF' with H_occupation_probability: the level's principal quantum number
   * (level_xion is its excitation energy), dissolved_only, its occupation
   * probability per cell */
  int occupation, dissolved_only, level_i, pad2;
  const double *level_w;
} or_bf_comp_t;

typedef struct or_cont_cells {
  const double *temp, *teta, *e_kT, *pe, *dxi, *ne;
  const double *nHI, *partHI, *nHeI, *nH2;
  double HI_xion;
  int helium_scattering, pad;
  const double *shield;  /* (1+a)^3.15/ne of compute_shield, for the H BF occupation levels */
} or_cont_cells_t;

/* load_lam_interp_weights: the stencils of one component on the wavelengths lam
 * (0-based iw, -1 where none); returns active, with fs/fe the first and last
 * wavelength with a stencil (0-based) */
int or_bf_weights(const or_bf_comp_t *c, int nlam, const double *lam, int *iw, unsigned char *quad, float *lagrange,
                  int *fs, int *fe);

/* continuum_opacities: xhat (nlam, ncell) set to the continuum's true absorption in
 * the working form, sigma (or NULL) to electron plus Rayleigh scattering; beta
 * (nlam, ncell) or NULL (boltzmann_factor from nu); 0 on success, -1 on an
 * unsupported component */
int or_continuum_opacities(int ncomp, const or_bf_comp_t *comps, int nlam, const double *lam, const double *nu,
                           int ncell, const or_cont_cells_t *cells, const float *beta, float *xhat, float *sigma);

/* init_H_levels with compute_shield (composition_mod.f90:2604-2613, 2708-2768):
 * shield (ncell), level_n and (with occupation) level_w (nk x ncell, level-major);
 * dissolve: the first cell's dxi > 0 without occupation probabilities */
void or_h_levels(int ncell, int nk, int occupation, const double *temp, const double *e_kT, const double *ne,
                 const double *dxi, const double *nHI, const double *nHeI, const double *partHI, double *shield,
                 double *level_n, double *level_w);

#ifdef __cplusplus
}
#endif
#endif

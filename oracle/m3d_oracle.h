/*
 * m3d_oracle.h -- CPU restatement of OpenMULTI3D's radiative-transfer hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA library is compared
 * against; it is never linked into, called by, or shipped with the product.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in the
 * build container, so the reference cannot be run here.  The restatement is
 * pinned by the reference's own in-source accuracy contracts (exp_neg /
 * linear_weights / parab_moments ulp bounds, QLG-bot max error against the
 * fp64 Humlicek-Weideman reference, window-extent guarantee) and by hand-derived
 * known answers; the end-to-end formal solution is otherwise "parity unpinned".
 *
 * Precision: every *_f32 routine follows the reference's real(4) arithmetic in
 * one fixed evaluation order (fused multiply-adds where marked, no other
 * contraction; the file is compiled with -ffp-contract=off).  The *_f64
 * routines are the plain FP64 truth with exact exp/expm1 forms.
 *
 * Array layout is the reference's own, Fortran column-major with frequency
 * fastest: work(f, x, y, z, k) with z = 0..nz+1 (one ghost plane each side).
 */
#ifndef M3D_ORACLE_H
#define M3D_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* formal solvers (rt_patch_mod.f90:1649-1721 selects among these) */
enum { OR_LINEAR = 0, OR_LINEAR2 = 1, OR_QUADRATIC = 2, OR_SHORT_LINEAR = 3, OR_SHORT_LINEAR2 = 4 };
/* upstream boundary modes (set_upstream_boundary, rt_patch_mod.f90:3270-3393) */
enum { OR_BND_NONE = 0, OR_BND_ZERO = 1, OR_BND_PCHIP = 2, OR_BND_LTE = 3 };

typedef struct {
  int nf, nx, ny, nz;        /* work is (nf, nx, ny, nz+2, 3) */
  int dir;                   /* +1 upward sweep (z increasing), -1 downward */
  int get_psi;               /* compute_psi */
  int split_rates;           /* rate_formulation == 'largest' */
  int pad;
  double ds[3];              /* cell size [cm] (ds * scaling%l) */
  double vec[3];             /* ray direction */
  double maser_dtau_max;     /* 2.0 default (m3d_patch_mod.f90:319) */
  double maser_Inu_max;      /* 1e30 default (m3d_patch_mod.f90:320) */
} or_slab_t;

/* ---- K0: exp / weights (exp_neg.inc, rt_solvers_mod.f90:785-877) ---- */
void or_exp_neg_f32(int n, const float *t, float *E, float *u0);
void or_exp4_f32(int n, const float *x, float *y);
void or_log_f32(int n, const float *x, float *y);
void or_linear_weights_f32(int n, const float *t, float *E, float *W, float *Psi, float *Esc);
void or_bezier3_weights_f32(int n, const float *t, float *w0, float *w1, float *w2, float *w3);
int or_long_char_hermite(const or_slab_t *s, float *work, float *psi, const float *beta, const float *pe,
                         const float *dpe_dz, const float *dlnt_dz, const float *temp, const float *hknu,
                         const float *g_pe, const float *g_dpe_dz, const float *g_dlnt_dz, const float *g_temp,
                         double code_length);
int or_long_char_hermite2(const or_slab_t *s, float *work, float *psi, const float *pe, const float *dpe_dz,
                          const float *g_pe, const float *g_dpe_dz, int ghost, double code_length);
int or_short_char_hermite(const or_slab_t *s, float *work, float *psi, float *irem, float *esc,
                          const float *beta, const float *pe, const float *dpe_dx, const float *dpe_dy,
                          const float *dpe_dz, const float *dlnt_dx, const float *dlnt_dy, const float *dlnt_dz,
                          const float *temp, const float *hknu, double code_length);
void or_linear_weights_f64(int n, const double *t, double *E, double *W, double *Psi, double *Esc);
void or_parab_moments_f32(int n, const float *t, float *E, float *U0, float *U1, float *q);
void or_parab_moments_f64(int n, const double *t, double *E, double *U0, double *U1, double *q);

/* ---- stencil (ray_mod.f90:493-597) ---- */
void or_set_stencil(const double ds[3], const double vec[3], double xkern[4], double ykern[4],
                    int *upo1, int *upo2, double *dsup);

/* ---- QLG (qlg_mod.f90) ---- */
void or_qlg_tables(float *tgx, float *th2x);               /* 9020 each, qlg_init */
void or_qlg_ref_f64(double a, double v0, double dv, int n, double *K);
void or_qlg_bot_sweep(const float *tgx, const float *th2x, float a, float v0, float dv, int n, float *K);
void or_qlg_bot_profile(const float *tgx, const float *th2x, int n, const float *a, const float *q,
                        const float *vpr, const float *idf, float *h);
int  or_qlg_bot_line_sweep(const float *tgx, const float *th2x, float D, float gL, float S, float ref,
                           float lnq, int nf, const double *llam, double llc, double pos, double idl,
                           float cap, int *fa, int *fb, float *hw, float *K);

/* ---- line opacity (linelist_mod.f90:729-960) ---- */
typedef struct {
  int nline;
  const double *llam0;      /* ln lambda0, ascending */
  const float *lower_ev, *gpref, *grad, *gw1, *gw2, *gstk;
  const uint8_t *unsold;    /* 1 -> Unsold van der Waals */
  const int *lev_i, *lev_j; /* NLTE levels (1-based, 0 = none), may be NULL */
  const uint8_t *active;    /* may be NULL (all active) */
  const float *reach_in;    /* per-line reach [log(lambda)] from a previous run, or NULL (has_reach = .false.) */
} or_linelist_t;

/* select_lines (linelist_mod.f90:1110-1142): the active lines whose reach window can
 * touch llam(1:nf) given the largest |vproj|; sel receives 0-based line indices in
 * ascending order, the return value is their number.  Without reach_in every active line. */
int or_select_lines(const or_linelist_t *ll, int nf, const double *llam, float vmax, int *sel);

/* per-cell fields (m1*m2*m3 cells, x fastest); cont, logref, chi, eta are (nf, cells) */
int or_add_opacity_equi(const float *tgx, const float *th2x, const or_linelist_t *ll,
                        int nf, const double *llam, int ncell,
                        float *chi, float *eta, const float *cont, const float *logref,
                        const float *vproj, const float *inv_df, const float *vbar2, const float *e_kT,
                        const float *lnbase, const float *ne, const float *tothi, const float *stark_pe,
                        const float *dep_mem, int nlevel, int do_nlte, float tol, float line_reject_frac,
                        uint8_t *used, float *strength, float *reach);
int or_add_opacity_equi_scat(const float *tgx, const float *th2x, const or_linelist_t *ll,
                             int nf, const double *llam, int ncell,
                             float *chi, float *eta, const float *cont, const float *logref,
                             const float *vproj, const float *inv_df, const float *vbar2, const float *e_kT,
                             const float *lnbase, const float *ne, const float *tothi, const float *stark_pe,
                             const float *dep_mem, int nlevel, int do_nlte, float tol, float line_reject_frac,
                             uint8_t *used, float *strength, float *reach, const float *one_m_eps,
                             float *chi_scat);

/* The plain FP64 line opacity (add_opacity_equi and QLG-bot in double, fp64 tables):
 * chl (nf, ncell) accumulated for one species, xhat (nf, ncell) and vproj in double */
void or_qlg_tables_f64(double *tgx, double *th2x);
int or_opacity_f64(const double *tgx, const double *th2x, const or_linelist_t *ll, int nf, const double *llam,
                   int ncell, double *chl, const double *xhat, const double *vproj, const float *inv_df,
                   const float *vbar2, const float *e_kT, const float *lnbase, const float *ne, const float *tothi,
                   const float *stark_pe, double tol);

/* ---- background and work units (rt_patch_mod.f90:1983-2023, 3518-3651) ---- */
void or_lte_background(int nf, int ncell, const double *nu, const float *temp, float *beta, float *Bnu);
void or_lte_work(int nf, int ncell, const float *chi_c, const float *beta, const float *Bnu,
                 float *xhat, float *ehat);
void or_logref(int n, const float *xhat, float tol, float *logref);
int  or_work_to_transfer_units(int nf, int ncell, float *w1, float *w2, const float *beta,
                               double maser_chi_floor, int suppress_masers);

/* ---- boundaries (rt_patch_mod.f90:3270-3393) ---- */
void or_upstream_boundary_f32(const or_slab_t *s, float *work, int mode, const float *mem,
                              float ds3_code, const float *ghost_r500, const float *ghost_temp,
                              const double *nu);
void or_upstream_boundary_f64(const or_slab_t *s, double *work, int mode, const double *mem,
                              float ds3_code, const float *ghost_r500, const float *ghost_temp,
                              const double *nu);

/* ---- rotate_array (rt_patch_mod.f90:3809-3866) ---- */
void or_rotate_array_f32(const or_slab_t *s, float *work, const double ds_code[3], double bot2pivot,
                         const double ray_offset[2]);
void or_rotate_array_f64(const or_slab_t *s, double *work, const double ds_code[3], double bot2pivot,
                         const double ray_offset[2]);

/* ---- formal solvers (rt_solvers_mod.f90) ---- */
int or_formal_solve_f32(int solver, const or_slab_t *s, float *work, float *psi, float *irem,
                        float *escape, const float *chi500, const float *chi500_up, const float *g500,
                        const int *eta_row, const uint8_t *eta_mask);
int or_formal_solve_f64(int solver, const or_slab_t *s, double *work, double *psi, double *irem,
                        double *escape, const float *chi500, const float *chi500_up, const float *g500,
                        const int *eta_row, const uint8_t *eta_mask);

/* ---- ALI accumulation (rt_patch_mod.f90:3399-3431) ---- */
void or_integrate_intensity(int nf, int ncell, float wmu, const float *work3, const float *psi,
                            float *Jnu, float *PsiJ);

/* ---- output (rt_patch_mod.f90:4151-4208) ---- */
void or_save_intensity(int nf, int nx, int ny, int nmu, const double *nu, const float *I_top,
                       const double *wmu, float *ie, float *flux);

#ifdef __cplusplus
}
#endif
#endif

/*
 * m3dgpu.h -- C ABI of libm3dgpu.so, the B200 (sm_100a) radiative-transfer hot
 * path of OpenMULTI3D: QLG-bot line opacity, the short- and long-characteristics
 * formal solvers, the ALI accumulation and the LTE synthesis output pass.
 *
 * Conventions follow HOP's libhop.h (experiments/OpenMULTI3D/HOP/standalone/
 * hop_c_api.f90:1-60):
 *   - every function returns an int status, 0 = ok, > 0 = error, and
 *     m3d_last_error(buf, len) gives the message;
 *   - arrays belong to the caller; nothing is retained after a call returns,
 *     except device buffers the library caches for its own scratch;
 *   - floating arrays are float32 (float64 with M3D_FP64), integer arrays int32;
 *   - multi-dimensional arrays use the reference's Fortran layout, first index
 *     fastest: work(f, x, y, z, k), frequency fastest.
 *
 * Host or device pointers: without M3D_DEVICE_PTRS every array is a host buffer
 * and the call copies it in and out synchronously; with M3D_DEVICE_PTRS every
 * array is a device pointer on the current device and the call is ordered on the
 * library stream (m3d_set_stream) and returns without synchronising.
 *
 * Thread safety: one context per host thread.  Each thread that calls the library
 * calls m3d_init first (and m3d_free before it exits); its context holds its own
 * stream, scratch and staging buffers, QLG tables, error string and counters, so
 * slabs handed to different host threads (the reference's OpenMP threads, one slab
 * each) run concurrently on their own streams.  libhop itself is one process-wide
 * instance; this library relaxes that.  Process-wide state: the loaded VCS tables
 * (m3d_vcs_load, guarded by a lock) and the no-allocation scratch array below.
 */
#ifndef M3DGPU_H
#define M3DGPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define M3D_OK 0
#define M3D_EINVAL 1      /* invalid argument */
#define M3D_ECUDA 2       /* CUDA runtime error */
#define M3D_ENOINIT 3     /* m3d_init has not been called */
#define M3D_EUNSUPPORTED 4
#define M3D_ENONFINITE 5  /* a non-finite value where the reference stops */

/* ---- flags ---- */
#define M3D_DEVICE_PTRS 0x1u  /* array arguments are device pointers */
#define M3D_FP64 0x2u         /* work/psi/irem/escape/mem are float64 (the plain FP64 path) */
#define M3D_GET_PSI 0x4u      /* compute the Lambda diagonal (rt_patch_t%compute_psi) */
#define M3D_SPLIT_RATES 0x8u  /* rate_formulation='largest': also Irem and escape */
#define M3D_LINE_DIAG 0x10u   /* accumulate the line diagnostics used/strength/reach */
#define M3D_ROTATE 0x20u      /* quadratic solver: apply rotate_array first (3D output pass) */
#define M3D_AUTOTUNE 0x40u    /* m3d_col_plan_create: time the launch shapes and keep the fastest */
#define M3D_COL_PERPOINT 0x80u /* m3d_col_plan_create: the per-point kernels instead of the fused column sweep */
#define M3D_SE_WARP 0x100u     /* m3d_stateq_update: one warp per cell whatever the atom's size */

/* ---- formal solvers (rt_patch_mod.f90:1649-1721, rt_params_mod.f90 solver names) ---- */
#define M3D_SOLVER_LINEAR 0        /* long_char_linear, rt_solvers_mod.f90:666 ('linear', 1D) */
#define M3D_SOLVER_LINEAR2 1       /* long_char2, rt_solvers_mod.f90:527 ('linear2', 1D) */
#define M3D_SOLVER_QUADRATIC 2     /* long_char_quadratic, rt_solvers_mod.f90:891 ('quadratic') */
#define M3D_SOLVER_SHORT_LINEAR 3  /* short_char, rt_solvers_mod.f90:19 ('linear', 3D) */
#define M3D_SOLVER_SHORT_LINEAR2 4 /* short_char2, rt_solvers_mod.f90:224 ('linear2', 3D) */

/* ---- upstream boundary (set_upstream_boundary, rt_patch_mod.f90:3270-3393) ---- */
#define M3D_BND_MEM 0    /* the upstream slab's exit plane, mem(f,x,y,1:3) */
#define M3D_BND_ZERO 1   /* top of the domain: no incoming radiation */
#define M3D_BND_PCHIP 2  /* bottom: pchip_mono extrapolation of planes 1..3, Inu = Snu */
#define M3D_BND_LTE 3    /* bottom: LTE ghost plane (lte_ghost) */

/* One depth slab of one ray direction: the state rt_patch_t carries into a sweep.
 * work is (nf, nx, ny, 0:nz+1, 3) with one ghost plane at each end. */
typedef struct m3d_slab {
  int nf, nx, ny, nz;
  int dir;            /* +1: sweep towards increasing z (upward rays), -1: downward */
  int get_psi;        /* also set by M3D_GET_PSI */
  int split_rates;    /* also set by M3D_SPLIT_RATES */
  int pad;
  double ds[3];       /* cell size [cm] (ds * scaling%l) */
  double vec[3];      /* ray direction, unit vector */
  double maser_dtau_max; /* nlte_params maser_dtau_max, default 2 (m3d_patch_mod.f90:319) */
  double maser_Inu_max;  /* nlte_params maser_Inu_max, default 1e30 (m3d_patch_mod.f90:320) */
} m3d_slab_t;

/* Line list of one isotope in structure-of-arrays form (line_types_mod.f90:22-75),
 * sorted ascending in llam0. */
typedef struct m3d_linelist {
  int nline;
  const double *llam0;          /* ln(lambda0 / AA) */
  const float *lower_ev;        /* lower level energy [eV] */
  const float *gpref;           /* loggf*ln10 + ln(bij_const/nu0) */
  const float *grad, *gw1, *gw2, *gstk; /* damping coefficients (bbtrans_mod.f90:78-106) */
  const unsigned char *unsold;  /* 1: Unsold van der Waals, 0: Barklem */
  const int *lev_i, *lev_j;     /* NLTE level indices, 1-based, 0 = LTE; may be NULL */
  const unsigned char *active;  /* may be NULL: every line active */
  const float *reach_in;        /* reach of a previous run [log(lambda)] (line_types_mod.f90:48-53),
                                   or NULL: has_reach = .false. */
} m3d_linelist_t;

/* ---- context (hop_init / hop_free / hop_last_error counterparts) ---- */
int m3d_init(int device, unsigned flags);
int m3d_free(void);
int m3d_last_error(char *buf, int buflen);
int m3d_version(int *major, int *minor, int *patch);
int m3d_set_stream(void *cuda_stream);        /* NULL: the library's own (non-blocking) stream;
                                                 cudaStreamLegacy: the legacy default stream */
int m3d_synchronize(void);
/* Number of kernel launches the library has issued since m3d_init. */
long long m3d_launch_count(void);

/* Device allocations and cached bytes of the calling thread's context: the number
 * of cudaMalloc calls the library has made for it, and the bytes its scratch and
 * host-staging caches hold.  No counterpart in the reference (a test hook that shows
 * which entry points allocate). */
int m3d_alloc_stats(long long *mallocs, unsigned long long *scratch_bytes, unsigned long long *staging_bytes);

/* Stage timing with CUDA events on the library stream (off by default).
 * Stages: 0 line opacity + transfer units, 1 formal solution (sweep), 2 intensity
 * reduction, 3 everything else.  m3d_profile_read synchronises and returns the
 * accumulated milliseconds and launch count of one stage since it was enabled. */
#define M3D_STAGE_OPACITY 0
#define M3D_STAGE_SOLVE 1
#define M3D_STAGE_REDUCE 2
#define M3D_STAGE_OTHER 3
int m3d_profile_enable(int on);
int m3d_profile_read(int stage, double *ms, long long *launches);

/* ---- K0: the transfer weights, elementwise over n points (diagnostics) ----
 * which: 0 exp_neg (E, u0), 1 linear_weights (E, W, Psi, Esc), 2 parab_moments
 * (E, U0, U1, q), 3 exp4 (y), 4 the library's fp32 log (y), 5 bezier3_weights
 * (w0, w1, w2, w3; rt_solvers_mod.f90:1280-1331).
 * Replaces exp_neg.inc:20-74 and rt_solvers_mod.f90:785-877. */
int m3d_weights(int which, int n, const void *t, void *o1, void *o2, void *o3, void *o4, unsigned flags);

/* ---- QLG-bot Voigt (qlg_mod.f90) ---- */
/* qlg_init (qlg_mod.f90:364-375): copies the two 9020-entry tables to the device. */
int m3d_qlg_init(void);
/* The tables as built, for inspection (host buffers of 9020 floats). */
int m3d_qlg_tables(float *tgx, float *th2x);
/* qlg_bot_profile (qlg_mod.f90:682-689), elementwise over n points. */
int m3d_qlg_bot_profile(int n, const float *a, const float *q, const float *vpr, const float *idf,
                        float *h, unsigned flags);

/* ---- line opacity: add_opacity_equi (linelist_mod.f90:729-960) ----
 * chi, eta, cont, logref are (nf, ncell); the per-cell fields are (ncell); dep_mem
 * is (ncell, nlevel).  chi and eta are accumulated in place.  used/strength/reach
 * (nline each) are updated with M3D_LINE_DIAG, else may be NULL.
 * With reach_in the lines are those select_lines keeps (linelist_mod.f90:1110-1142:
 * centres within the chunk widened by half a grid step, max |vproj| and each line's
 * reach), and lines centred beyond the chunk take the unfloored reference at the
 * nearer end and a window capped by their reach (:844-854, 914-921).  The LTE
 * scattering split is m3d_line_opacity_scat. */
int m3d_line_opacity(const m3d_linelist_t *ll, int nf, const double *llam, int ncell,
                     float *chi, float *eta, const float *cont, const float *logref,
                     const float *vproj, const float *inv_df, const float *vbar2, const float *e_kT,
                     const float *lnbase, const float *ne, const float *tothi, const float *stark_pe,
                     const float *dep_mem, int nlevel, int do_nlte, float tol, float line_reject_frac,
                     unsigned char *used, float *strength, float *reach, unsigned flags);
/* add_opacity_equi with line_scattering (do_scat, linelist_mod.f90:933-939): every
 * LTE line (not a departure-carrying one) also adds one_m_eps times its profile to
 * chi_scat, both (nf, ncell) like chi, chi_scat accumulated in place, in line order.
 * The caller forms one_m_eps per stage (compute_epsilon_stage) and folds chi_scat
 * into the source (work_to_transfer_units' chi_scat*dJnu, m3d_lte_emission's dJnu). */
int m3d_line_opacity_scat(const m3d_linelist_t *ll, int nf, const double *llam, int ncell,
                          float *chi, float *eta, const float *cont, const float *logref,
                          const float *vproj, const float *inv_df, const float *vbar2, const float *e_kT,
                          const float *lnbase, const float *ne, const float *tothi, const float *stark_pe,
                          const float *dep_mem, int nlevel, int do_nlte, float tol, float line_reject_frac,
                          unsigned char *used, float *strength, float *reach, const float *one_m_eps,
                          float *chi_scat, unsigned flags);

/* add_linelist_opacities' last step with line scattering (composition_mod.f90:1864-1874):
 * chi_scat *= 1 - beta over n points, after every species has been added. */
int m3d_chi_scat_units(long long n, float *chi_scat, const float *beta, unsigned flags);

/* ---- background and work units ---- */
/* beta = max(exp(-h nu/kT), tiny), Bnu = beta/(1-beta): (nf, ncell)
 * (lte_background_opacities, rt_patch_mod.f90:2004-2023) */
int m3d_lte_background(int nf, int ncell, const double *nu, const float *temp, float *beta,
                       float *Bnu, unsigned flags);
/* (xhat, ehat) -> (chi, Snu) in place, maser floor (work_to_transfer_units,
 * rt_patch_mod.f90:3571-3651, without split rates or line scattering).
 * n_floored (may be NULL) receives the number of floored points. */
int m3d_work_to_transfer_units(int nf, int ncell, float *w1, float *w2, const float *beta,
                               double maser_chi_floor, int suppress_masers, int *n_floored,
                               unsigned flags);

/* ---- formal solution of one slab (radiative_transfer, rt_patch_mod.f90:1649) ----
 * psi, irem, escape are (nf, nx, ny, nz); chi500, chi500_up (this direction) are
 * (nx, ny, nz) and g500 the ghost plane's chi500 (nx, ny) -- the linear2 solvers
 * only.  eta_row (nx, ny, nz; 0 = no flags) and eta_mask (nf, nrows) are the
 * update_eta_mask flags, may be NULL.  With M3D_ROTATE the quadratic solver first
 * applies rotate_array to work(:,:,:,1:nz,1:2), which then holds the sheared
 * chi and Snu as in the reference; rot_ds_code, rot_bot2pivot, rot_offset are
 * rotate_array's cell size [code units], pivot height above the slab bottom and
 * ray_offset [cells].  The short-characteristics solvers need the upwind point
 * within one cell horizontally, |vec[0]/vec[2]| ds[2] <= ds[0] and the same in y
 * (set_stencil, ray_mod.f90:493-512); other directions return M3D_EINVAL. */
int m3d_formal_solve(int solver, const m3d_slab_t *slab, void *work, void *psi, void *irem,
                     void *escape, const float *chi500, const float *chi500_up, const float *g500,
                     const int *eta_row, const unsigned char *eta_mask, const double *rot_ds_code,
                     double rot_bot2pivot, const double *rot_offset, unsigned flags);

/* ---- long_char_hermite (rt_solvers_mod.f90:1052-1504), the optional 'hermite'
 * solver: chain-rule cubic-Hermite long characteristics along z for one slab of
 * at least 3 planes, FP32.  work (nf, nx, ny, 0:nz+1, 3) holds chi, Snu and the
 * upstream ghost plane (m3d_upstream_boundary); Inu is written to slot 3 and, with
 * slab->get_psi, the Lambda diagonal per chi to psi (nf, nx, ny, nz).  The ghost's
 * thermodynamic state (the model below the bottom, or an upstream neighbour's
 * exit plane) takes the full step; without it (all ghost_* NULL) the first plane
 * takes herm_first's secant step from the zeroed top ghost. */
typedef struct {
  const float *beta;                                   /* (nf, nx, ny, nz): exp(-h nu/kT) */
  const float *pe, *dpe_dz, *dlnt_dz, *temp;           /* (nx, ny, nz): Pe, dPe/dz, dlnT/dz, T */
  const float *hknu;                                   /* (nf): h nu / k */
  const float *ghost_pe, *ghost_dpe_dz, *ghost_dlnt_dz, *ghost_temp; /* (nx, ny), or NULL */
  double code_length;                                  /* cm per length unit of the d/dz (scaling%l) */
} m3d_hermite_t;
int m3d_long_char_hermite(const m3d_slab_t *slab, float *work, float *psi, const m3d_hermite_t *h,
                          unsigned flags);

/* ---- long_char_hermite2 (rt_solvers_mod.f90:1536-1895), the optional 'hermite2'
 * solver: dtau by long_char_hermite's chain rule (control points bounded by
 * 3 |secant|), the source by long_char_quadratic's parabola with dS/dtau at the
 * target MC-limited from the two adjacent intervals; dtau, 1/dtau and the weights
 * in FP64 as the reference declares them.  One slab of at least 2 planes, FP32;
 * work and psi as m3d_long_char_hermite.  pe, dpe_dz (nx, ny, nz); ghost selects
 * the upstream ghost's Pe: 0 the zeroed top ghost (ghost_* NULL; herm2_first's
 * secant step), 1 an upstream neighbour's exit plane, 2 the model below the bottom
 * (ghost_pe, ghost_dpe_dz (nx, ny)); 1 and 2 differ only for nz == 2, where the
 * last plane's third sample is the ghost and only a neighbour supplies its Pe. */
int m3d_long_char_hermite2(const m3d_slab_t *slab, float *work, float *psi, const float *pe, const float *dpe_dz,
                           const float *ghost_pe, const float *ghost_dpe_dz, int ghost, double code_length,
                           unsigned flags);

/* ---- short_char_hermite (rt_solvers_mod.f90:1917-2248), the chain-rule Hermite
 * short characteristics ('hermite' on the 3D iteration path), FP32: short_char's
 * 4x4 upwind kernels and 2x2 minimum, also over chi/Pe and Snu/Bnu formed at the
 * upwind nodes, and the quadratic weights with product-rule slopes along the ray
 * (directional derivatives from the x/y/z partials); dtau and the weights in FP64
 * as the reference declares them.  The first plane takes short_char's linear
 * step.  work, psi, irem, escape as m3d_formal_solve's short characteristics
 * (periodic x/y, the same stencil precondition); irem/escape with split_rates. */
typedef struct {
  const float *beta;                                   /* (nf, nx, ny, nz): exp(-h nu/kT) */
  const float *pe, *dpe_dx, *dpe_dy, *dpe_dz;          /* (nx, ny, nz): Pe and its partials */
  const float *dlnt_dx, *dlnt_dy, *dlnt_dz, *temp;     /* (nx, ny, nz): ln T partials, T */
  const float *hknu;                                   /* (nf): h nu / k */
  double code_length;                                  /* cm per length unit of the partials */
} m3d_hermite3d_t;
int m3d_short_char_hermite(const m3d_slab_t *slab, float *work, float *psi, float *irem, float *escape,
                           const m3d_hermite3d_t *h, unsigned flags);

/* ---- sampled opacity tables (HOP/optab_mod.f90:37-166, :181-409): an opacity
 * per unit chi500 on (wavelength, PC axis 1, PC axis 2) of (ln T, ln ne), held
 * resident on the device with its monotone node slopes and sampled per
 * (frequency, cell) by a separable cubic Hermite.  rot is pca_transform_type's
 * rot(2,2) in Fortran order: rot(1,1), rot(2,1), rot(1,2), rot(2,2). */
typedef struct {
  double mu[2];     /* mean of (ln T, ln ne) */
  double rot[4];    /* PC directions, columns */
  double c0[2];     /* first node coordinate along each PC axis */
  double dc[2];     /* node spacing along each PC axis */
} m3d_pca_t;
typedef struct m3d_optab m3d_optab_t;
/* sample_optab_type with sample_build_derivatives: val, scat (nnu, ntemp, nne),
 * wavelength fastest, over the ascending nodes lam (nnu) [A]; scat may be NULL
 * (a line-list table without line scattering).  Needs nnu, ntemp, nne >= 2. */
int m3d_optab_create(int nnu, int ntemp, int nne, const double *lam, const float *val, const float *scat,
                     const m3d_pca_t *pca, unsigned flags, m3d_optab_t **out);
/* the node slopes along wavelength, PC axis 1 and PC axis 2 (dl, dt, de; or sl,
 * st, se for component 1), (nnu, ntemp, nne) each */
int m3d_optab_slopes(const m3d_optab_t *t, int component, float *dl, float *dt, float *de, unsigned flags);
/* sample_interpolate: per cell temp, ne (fp64) and chi500; the frequencies' vacuum
 * wavelengths lam_q (nf); back = total extinction, scat = its scattering part,
 * (nf, ncell) frequency fastest, set.  The table needs its scattering component. */
int m3d_optab_sample(const m3d_optab_t *t, long long ncell, const double *temp, const double *ne, const float *chi500,
                     int nf, const double *lam_q, float *back, float *scat, unsigned flags);
/* sample_interpolate_ll: the query wavelength of a cell is lam_q (1 + vproj);
 * xhat and ehat (nf, ncell) += kappa chi500 (pass the two work slots); chi_scat
 * (nf, ncell) += the scattering component's kappa chi500 when it and the table's
 * scattering component are both given. */
int m3d_optab_sample_ll(const m3d_optab_t *t, long long ncell, const double *temp, const double *ne,
                        const float *chi500, const float *vproj, int nf, const double *lam_q, float *xhat,
                        float *ehat, float *chi_scat, unsigned flags);
int m3d_optab_destroy(m3d_optab_t *t);

/* ---- hydrogen line profiles (HOP/hprofl_mod.f90, after HLINOP), the analytic path:
 * Griem's Stark profile with the VCS-approximating corrections and the Holtsmark
 * ion field, QLG-bot Voigt profiles over the fine-structure components, Lyman
 * alpha's quasi-molecular satellite wings.  hline_t (hprofl_mod.f90:156-165): */
typedef struct {
  int n, m, bpo, io;                  /* lower and upper level, BPO self-broadening, components */
  int opts, pad;                      /* the M3D_H_* switches it was built with */
  double nu0, grad, gstk, gw1, gw2, gw3;
  double dq[14], wt[14];              /* fine-structure offsets [nu/nu0] and weights */
  double dqbar, dqmax, qray;
} m3d_hline_t;
/* the per-cell inputs of add_h_opacities (float, ncell each): projected velocity
 * [v/c], inverse Doppler width c/v_th, T, lower-level density, ne, neutral H,
 * mean relative speed squared with H, Holtsmark normal field, (T/1e4)^0.3 n(He) */
typedef struct {
  const float *vproj, *inv_df, *temp, *ni, *ne, *tothi, *vbar2h, *fo, *t3nhe;
} m3d_hcells_t;
#define M3D_H_NO_RAD 1u    /* disable_rad */
#define M3D_H_NO_STARK 2u  /* disable_stk */
#define M3D_H_NO_VDW 4u    /* disable_vdw */
#define M3D_H_NO_BPO 8u    /* hydrogen_BPO = .false. */
/* The tabulated profiles of HOP/hvcs_mod.f90 (read_vcs_grid): load one series'
 * table file (1 Balmer, 2 Paschen, 3 Brackett; radiative = the table includes
 * radiative damping), as hydrogen_profiles = 'stehle' or 'lemke' selects them.
 * While a line's series holds its (n, m), its profile is the table's, with the
 * missing broadening added as a Lorentzian; otherwise the analytic one. */
int m3d_vcs_load(int series, const char *path, int radiative);
int m3d_vcs_clear(void);
int m3d_vcs_supported(int n, int m);   /* 1 when the loaded tables hold the line */
/* hydrogen_line (hprofl_mod.f90:703-810): the line's widths and fine structure, on the host */
int m3d_hydrogen_line(int n, int m, double nu0, unsigned opts, m3d_hline_t *h);
/* hcell_prepare + hprofile per cell at nq detunings q = (nu - nu0)/nu0: phi (ncell, nq), q fastest */
int m3d_h_profile(const m3d_hline_t *h, long long ncell, const m3d_hcells_t *cells, int nq, const double *q,
                  float *phi, unsigned flags);
/* add_h_opacities (hprofl_mod.f90:208-385): from the line-centre index f0 (0-based)
 * outwards in both directions until the line opacity falls below 1e-7 of cont at f0
 * in each cell, chi += phi R bi, eta += phi R bj with R = ni Bij (bi = bj = NULL in
 * LTE); chi, eta, cont (nf, ncell).  line_used and line_strength are raised. */
int m3d_h_opacity(const m3d_hline_t *h, double Bij, int f0, int nf, const double *nu, long long ncell,
                  const m3d_hcells_t *cells, const float *bi, const float *bj, float *chi, float *eta,
                  const float *cont, int *line_used, float *line_strength, unsigned flags);

/* ---- output files: patch_t%save5 (tasks/patch_mod.f90:4248-4346) from the library's
 * buffers.  Writes <run_dir>/save/<label>_<key>.bin, the float32 array of shape dims
 * (5, Fortran order, first fastest) raw, and with add2meta appends its line to
 * <label>_meta.txt (header on creation).  key: 1 to 3 integers (abs, 3 digits each),
 * as patch_t%key(1:3) or (1:2).  mem is a host pointer, or a device pointer with
 * M3D_DEVICE_PTRS.  save_intensity's 'ie' (nf,1,1,nmu,nset) and 'flux' (nf,1,1,1,nset),
 * and the J/PsiJ/Jali of rt_to_file, are such arrays. */
int m3d_save5(const char *run_dir, const char *label, const int *key, int nkey, const float *mem, const int *dims,
              int add2meta, unsigned flags);

/* rotate_array (rt_patch_mod.f90:3809-3866) on work(:,:,:,1:nz,1:2), in place. */
int m3d_rotate_array(const m3d_slab_t *slab, void *work, const double *ds_code, double bot2pivot,
                     const double *ray_offset, unsigned flags);

/* m3d_rotate_array for callers that cannot let the library allocate device memory:
 * programs whose own pool holds all device memory, or whose other streams must not
 * stall on the device-wide synchronisation of cudaMalloc/cudaFree.
 * It has no counterpart in the reference.  It allocates nothing: its scratch is one
 * fixed 8 MiB array inside the library's device image, held by every GPU that loads
 * the library until the process exits, so one plane (nf*nx*ny values of the chosen
 * precision) may use at most 8 MiB; larger slabs are rejected with M3D_EINVAL.
 * work must be a device pointer (M3D_DEVICE_PTRS is required; M3D_FP64 optional).
 * Every call looks up the array's device address on the context's device
 * (cudaGetSymbolAddress, which allocates nothing); make the first call on a device
 * before any stream capture.  The array is one per device, shared by all calls and
 * all host threads' contexts: calls that overlap on the GPU (different streams or
 * threads at the same time) race, so serialise them.  Each call overwrites the
 * scratch before reading it, so nothing in it has to start at zero.  Results are
 * bit-identical to m3d_rotate_array. */
int m3d_rotate_array_noalloc(const m3d_slab_t *slab, void *work, const double *ds_code, double bot2pivot,
                             const double *ray_offset, unsigned flags);

/* set_upstream_boundary (rt_patch_mod.f90:3270-3393): fills the ghost plane of work.
 * mem is (nf, nx, ny, 3) for M3D_BND_MEM; ghost_r500 = chi500_ghost/chi500(:,:,1)
 * and ghost_temp (nx, ny) plus nu (nf) for M3D_BND_LTE; ds3_code is ds(3) in code
 * units for M3D_BND_PCHIP. */
int m3d_upstream_boundary(const m3d_slab_t *slab, void *work, int mode, const void *mem,
                          float ds3_code, const float *ghost_r500, const float *ghost_temp,
                          const double *nu, unsigned flags);

/* ---- ALI accumulation: integrate_intensity (rt_patch_mod.f90:3399-3431) ----
 * Jnu += 2 wmu I, PsiJ += 2 wmu Psi over n points (PsiJ, psi may be NULL). */
int m3d_integrate_intensity(int n, float wmu, const float *inu, const float *psi, float *Jnu,
                            float *PsiJ, unsigned flags);

/* ---- LTE synthesis output pass of one frequency window ----
 * The whole do_final branch of rt_patch_t%execute (rt_patch_mod.f90:1014-1030)
 * for every direction and every depth slab of the column, bottom slab first:
 * LTE background, line opacity of every species (add_linelist_opacities,
 * composition_mod.f90:1663-1954), work_to_transfer_units, the bottom PCHIP ghost,
 * rotate_array and long_char_quadratic with the exit plane handed from slab to
 * slab, then save_intensity (rt_patch_mod.f90:4151-4208).
 */
typedef struct m3d_species {
  m3d_linelist_t ll;
  const float *inv_df;  /* (ncell) inverse Doppler factor c/v (ion_mod.f90:198) */
  const float *vbar2;   /* (ncell) compute_vbar2 (ion_mod.f90:214) */
  const float *lnbase;  /* (ncell) ln n - ln U + ln inv_df (linelist_mod.f90:1042-1047) */
} m3d_species_t;

typedef struct m3d_atmos {
  int nx, ny, nz;          /* cells; plane z = 1 is the bottom of the domain */
  int nslab;               /* depth slabs, bottom first */
  const int *slab_nz;      /* planes per slab (nslab), each >= 2, summing to nz (host memory) */
  double ds_cm[3];         /* cell size [cm] */
  double ds_code[3];       /* cell size [code units], for rotate_array */
  double pivot_z;          /* pivot height above the bottom of the domain [code units] */
  double ray_offset[2];    /* [cells] */
  const float *temp;       /* (ncell) [K] */
  const float *chi_c;      /* (ncell) grey continuum extinction [1/cm], pure absorption */
  const float *vx, *vy, *vz; /* (ncell) velocity [c] */
  const float *e_kT, *ne, *tothi, *stark_pe; /* (ncell) */
  int nspecies;
  const m3d_species_t *species; /* host memory; the arrays inside follow M3D_DEVICE_PTRS */
  double tol;              /* linelist_params tolerance, 1e-4 */
  double maser_chi_floor;  /* 1e-4 */
  double maser_dtau_max;   /* 2 */
  double maser_Inu_max;    /* 1e30 */
} m3d_atmos_t;

/* nu (nf) [Hz], llam (nf) = ln(lambda/AA), uniform; vec (3, nray) (host), wmu (nray)
 * flux weights (host).  Outputs: i_top (nf, nx, ny, nray) the emergent intensity in
 * transfer units (may be NULL), ie (nf, nray) and flux (nf) as save_intensity writes
 * them.  With M3D_FP64 the whole pass runs in FP64 (the plain FP64 path): the line
 * opacity and its QLG-bot profile with fp64 tables, exp and log, the transfer units,
 * and rotate_array + the quadratic solver one launch per ray and slab; i_top is then
 * float64. */
/* The opacity stage of m3d_lte_synthesis for one direction vec (3, host): the
 * background (beta, Bnu), work units, add_opacity_equi of every species in line
 * order with the Doppler shift v.vec, and work_to_transfer_units (rt_patch_mod.f90:
 * 2004-2023, 3518-3536, 3571-3651; linelist_mod.f90:729-960).  Outputs chi and S
 * (nf, ncell), frequency fastest, cell index x fastest then y then z; float64 with
 * M3D_FP64 (the plain FP64 path). */
int m3d_lte_transfer_units(const m3d_atmos_t *atm, int nf, const double *nu, const double *llam, const double *vec,
                           void *chi, void *S, unsigned flags);

int m3d_lte_synthesis(const m3d_atmos_t *atm, int nf, const double *nu, const double *llam,
                      int nray, const double *vec, const double *wmu, void *i_top, float *ie,
                      float *flux, unsigned flags);

/* m3d_lte_synthesis over nwin windows of nf = 32 frequencies in one call, the
 * reference's n_windows loop (ray_patch_mod.f90:97-127) with its windows on the
 * device at once: nu and llam (nwin x nf) hold the windows one after the other, each
 * window's grid formed from its own frequencies; ie (nray, nwin nf), flux (nwin nf),
 * i_top (nray, ny, nx, nwin nf).  Equal bit for bit to one m3d_lte_synthesis call per
 * window.  For atmospheres too small to fill the GPU with one window (a 1D column of
 * 80 depths is three warps per window), where it runs the opacity of every ray and
 * window in one launch; the transfer units of all rays and windows are held at once
 * (8 B per ray, cell and frequency of the batch; 16 B with M3D_FP64).  No reach_in. */
int m3d_lte_synthesis_windows(const m3d_atmos_t *atm, int nwin, int nf, const double *nu, const double *llam,
                              int nray, const double *vec, const double *wmu, void *i_top, float *ie,
                              float *flux, unsigned flags);

/* ---- libhop's opacity call ----
 * m3d_hop_set_state loads a state for m3d_hop_opacity (host copies; the calling
 * thread's; velocities, slabs and geometry are ignored): the cells' e_kT, ne, tothi,
 * stark_pe and every species' line list with its inv_df, vbar2 and lnbase, the
 * roles hop_load_state and hop_init_linelist play for libhop.
 * m3d_hop_opacity has hop_opacity's argument list (HOP/standalone/libhop.h:20,
 * hop_c_api.f90:910-942) with host buffers, so that libhop's hop_opacity can forward
 * its line-list part unchanged: lam vacuum AA ascending and uniform in ln(lambda)
 * (constant R); chi (nlam, n) holds the caller's continuum + absmet on entry, which
 * is the tolerance reference, and gets the line list added as add_linelist_opacities
 * adds it (composition_mod.f90:1663-1954: a line accumulator from zero, every
 * species in turn, the lines within line_margin [AA] of the grid); scat is left
 * alone.  include_absmet must be 0 (the continuum is the caller's), line_scat must be
 * <= 0 (the scattering split needs HOP's epsilon per stage), include_llist = 0 does
 * nothing. */
int m3d_hop_set_state(const m3d_atmos_t *atm);
int m3d_hop_free_state(void);
int m3d_hop_opacity(int nlam, const double *lam, float *chi, float *scat, int include_absmet, int include_llist,
                    double line_margin, int line_scat);

/* Gradients of the LTE pass, accumulated (+=) by m3d_lte_synthesis_adjoint.  Cell
 * arrays (ncell, x fastest); per-species arrays species-major; gpref the species'
 * line lists one after the other.  Pointers follow M3D_DEVICE_PTRS. */
typedef struct m3d_lte_grad {
  float *temp;    /* (ncell) dL/dtemp through the LTE background (beta, Bnu) only */
  float *chi_c;   /* (ncell) dL/dchi_c */
  float *e_kT;    /* (ncell) dL/de_kT (the Boltzmann factors of every species) */
  float *inv_df;  /* (nspecies, ncell) dL/dinv_df (the Doppler width in the profile and in S) */
  float *lnbase;  /* (nspecies, ncell) dL/dlnbase */
  float *gpref;   /* (sum of nline) dL/dgpref: gpref = log gf ln 10 + const, so this is dL/dlog gf / ln 10 */
} m3d_lte_grad_t;

/* The reverse mode of m3d_lte_synthesis for one window of 32 frequencies and every
 * ray: given g_flux = dL/dflux (nf), adds dL/d(input) into grad.  No counterpart in
 * the reference (its abundance fits take finite differences of whole syntheses,
 * tumult/abundance.py).  Stage by stage, backwards: save_intensity; the fused
 * rotate_array + long_char_quadratic sweep reversed per column from intensities
 * checkpointed at the slab faces; the transpose of rotate_array; the transfer units;
 * add_opacity_equi's line loop replayed with the forward's decisions.  Window
 * limits, tolerance tests, limiter branches and clamps are held as the forward takes
 * them.  QLG-bot snaps to the nearest table node; its derivative is that of the
 * continuous member (G(u) = 2^-u, W'(u) from the table's differences).  Damping,
 * velocities, ne and tothi are held fixed.  Slabs of at most 64 planes, at most 64
 * slabs, no reach_in; the FP32 pass only. */
int m3d_lte_synthesis_adjoint(const m3d_atmos_t *atm, int nf, const double *nu, const double *llam, int nray,
                              const double *vec, const double *wmu, const float *g_flux, const m3d_lte_grad_t *grad,
                              unsigned flags);

/* ---- continuum opacity of a window: composition_type%continuum_opacities
 * (HOP/composition_mod.f90:2893-2984) -- the H I levels above n = 15 (add_hrest,
 * :3807-3846), every absdat component (bftrans_mod.f90: load_lam_interp_weights
 * :100-198, absorption_factor :476-531, interp_xkap :235-452), the components tabulated
 * with stimulated emission over 1 - beta, and the scattering opacity: electrons
 * (:3851-3872) and Rayleigh by H I, H2 and He I (:3878-3939).  The EOS state and the
 * components' tables are inputs. */
#define M3D_BF_HMINUS 1    /* 'H- BF': n */
#define M3D_BF_NPE 2       /* 'H- FF', 'H2-', 'HE-': n Pe */
#define M3D_BF_H 3         /* 'H BF': 2.0898e-26/(2 k^5) n_k, or wcalc2 under occupation probabilities */
#define M3D_BF_H_FF 4      /* 'H FF': 2.0898e-26 kT/(2 Ryd) n exp(-(xion - dxi)/kT) / U */
#define M3D_BF_PAIR 5      /* 'H+H', 'H+HE', 'H2+H', 'H2+H2', 'H2+HE': n n2 */
#define M3D_BF_H2PLUS 6    /* 'H2+': 1e-40 n n2 */
#define M3D_BF_PEDEP 7     /* a Pe-dependent table: n Pe */
#define M3D_BF_PEACH 8     /* a Pe-dependent Peach table: 1e-40/e e_kT n Pe */
#define M3D_BF_MOLECULAR 9 /* n awgt / N_A, the mass density */
#define M3D_BF_REGULAR 10  /* a level's bound-free: g exp(-xion/kT) n / U */

/* One absdat component (bftrans_type).  Tables are host memory: lam (nnu) [AA],
 * lnlam (nnu, with loglam), tt (ntt) the temperature nodes (T [K], or 5040/T with
 * iteta), xkap (nnu x ntt, wavelength fastest) as set_table stores it (divided by
 * xkap_scale, logarithmic when log_table), ldisk (nnu).  The per-cell arrays (ncell,
 * float64) follow the call's flags: n the particle's number density [cm^-3]; n2 the
 * second particle's (pairs, H2+); part the particle's ln partition function (H FF,
 * regular); level_n the population of H I level k (M3D_BF_H).
 * occupation: an 'H BF' level under H_occupation_probability (the reference's
 * default): a table without temperature dependence goes through wcalc2
 * (level_mod.f90:149-279) with level_i the level's principal quantum number,
 * level_xion its excitation energy [eV], level_n its population, level_w its
 * occupation probability (per cell), n H I's number density, and the cells' ne, nHeI
 * and shield; dissolved_only leaves out the wavelengths beyond the series limit.
 * With temperature nodes the level keeps absorption_factor's huge(1d0) factor, as
 * the reference does. */
typedef struct m3d_bf_comp {
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
  int occupation, dissolved_only, level_i, pad2;
  const double *level_w;
} m3d_bf_comp_t;

/* The EOS state of the cells (ncell, float64, per the call's flags): temp [K], teta
 * = 5040/T, e_kT = 1 eV/kT, pe [dyn cm^-2], dxi the ionisation-energy lowering [eV],
 * ne [cm^-3]; H I's number density and ln partition function (the H rest; NULL: no
 * H rest, no H I Rayleigh), He I and H2 densities (Rayleigh; may be NULL), H I's
 * ionisation energy [eV], and helium_scattering (the reference's switch, default on);
 * shield = (1+a)^3.15/ne of compute_shield (composition_mod.f90:2604-2613) [cm^3],
 * for the H BF levels under occupation probabilities (else may be NULL). */
typedef struct m3d_cont_cells {
  const double *temp, *teta, *e_kT, *pe, *dxi, *ne;
  const double *nHI, *partHI, *nHeI, *nH2;
  double HI_xion;
  int helium_scattering, pad;
  const double *shield;
} m3d_cont_cells_t;

/* xhat (nlam, ncell) = the continuum's true absorption in the working form (the
 * components in order; those with istim summed apart and divided by 1 - beta);
 * sigma (nlam, ncell, may be NULL) = electron + Rayleigh scattering [1/cm].  lam and
 * nu (nlam, host) are the window's wavelengths [AA] and frequencies [Hz]; beta
 * (nlam, ncell) or NULL, then boltzmann_factor from nu. */
int m3d_continuum_opacities(int ncomp, const m3d_bf_comp_t *comps, int nlam, const double *lam, const double *nu,
                            int ncell, const m3d_cont_cells_t *cells, const float *beta, float *xhat, float *sigma,
                            unsigned flags);

/* The H I level set-up the continuum's 'H BF' components read, init_H_levels with
 * compute_shield (composition_mod.f90:2604-2613, 2708-2768) over ncell cells (float64,
 * per the flags): shield (ncell) = (1 + 0.08989 ne^0.16667/sqrt(T))^3.15 / ne; for the
 * hydrogenic levels i = 1..nk (nk <= 100) level_n (nk x ncell, level-major: level_n[c +
 * ncell (i-1)]) = nHI g_i exp(-e_kT Ryd (1 - 1/i^2)) part.  With occupation (the
 * reference's H_occupation_probability) level_w (same layout) = wcalc's occupation
 * probability of each level (level_mod.f90:108-142, from nHI, nHeI, ne and shield) and
 * part = 1/sum_i w_i g_i exp(..); without, part = exp(-partHI) and, when the first cell
 * has dxi > 0 (as the reference decides), the levels above n = sqrt(Ryd/dxi) of each
 * cell dissolved (a cell with dxi <= 0 keeps them all); level_w and nHeI may be NULL. */
int m3d_h_levels(int ncell, int nk, int occupation, const double *temp, const double *e_kT, const double *ne,
                 const double *dxi, const double *nHI, const double *nHeI, const double *partHI, double *shield,
                 double *level_n, double *level_w, unsigned flags);

/* composition_type%opacity (composition_mod.f90:3122-3260), the whole pipeline that
 * hop.opacity() and chi500 call, over ncell cells (those of the loaded state with
 * include_llist): beta (the caller's (nlam, ncell), or NULL: boltzmann_factor from nu
 * and cells->temp);
 * continuum_opacities of the components and cells (m3d_continuum_opacities) into the
 * working xhat and the scattering opacity; with include_llist the line list of the
 * state, the lines within line_margin [AA], against that xhat as the tolerance
 * reference (as m3d_hop_opacity adds it, no velocities); then the one conversion to
 * physical extinction, chi = xhat - ehat beta (the continuum alone: xhat (1 - beta)),
 * plus the scattering opacity unless disjoint.  scat (or NULL) = electron + Rayleigh
 * scattering.  lam (nlam) [AA] ascending (uniform in ln(lambda) with the line list,
 * nlam >= 2 then), nu (nlam) [Hz]; chi, scat (nlam, ncell); host buffers.  No absmet,
 * no line scattering split (the reference's include_absmet and line_scat off).
 * chi500, load_state_variables' reference opacity (composition_mod.f90:2169-2176), is
 * this call at the one vacuum wavelength of 5000 A air without the line list. */
int m3d_opacity(int nlam, const double *lam, const double *nu, int ncell, int ncomp, const m3d_bf_comp_t *comps,
                const m3d_cont_cells_t *cells, const float *beta, float *chi, float *scat, int include_llist,
                double line_margin, int disjoint);

/* ---- statistical equilibrium (FP64) ----
 * Level and transition indices are 0-based (the reference's minus one).  Per-cell
 * arrays keep the cell index fastest: b(cell, level) at b[cell + ncell*level], as
 * adata%b(x,y,z,level) with cell = x + nx*(y + ny*z).  The atom tables are host
 * memory whatever the flags; M3D_DEVICE_PTRS applies to the per-cell arrays, those an
 * m3d_col_cells_t points to included (the struct itself is host memory). */
#define M3D_SE_LINEQ_NO_PIVOT 0 /* lse_solver='lineq_no_pivot' (default; 'eqsyst' rounds identically) */
#define M3D_SE_LINEQ 1          /* lse_solver='lineq': full pivoting */
#define M3D_SE_LU_PARTIAL 2     /* LU with partial (row) pivoting */
#define M3D_COL_REGEMORTER 1    /* e_excitation='regemorter' (atom_mod.f90:1825-1832) */
#define M3D_COL_SEATON 2        /* e_ionisation='seaton' (atom_mod.f90:1814-1822) */
#define M3D_COLH_DRAWIN 1       /* h_excitation / h_ionisation='drawin' (atom_mod.f90:1861-1871) */
#define M3D_COLH_TAKEDA 2       /* h_forbidden='takeda', a pair without a line (atom_mod.f90:1856-1860) */

/* gencol's record kinds (atom_mod.f90:2288-2344) */
#define M3D_GENCOL_NONE 0       /* a named collider the composition lacks: no rate */
#define M3D_GENCOL_OHM 1        /* 'OHM', 'OHMEGA': electrons on positive ions, a collision strength */
#define M3D_GENCOL_CE 2         /* 'CE': electron excitation of neutrals */
#define M3D_GENCOL_CH 3         /* 'CH': bound-bound with neutral hydrogen, a downward rate */
#define M3D_GENCOL_CHI 4        /* 'CHI': bound-free with neutral hydrogen, an upward rate */
#define M3D_GENCOL_CI 5         /* 'CI': electron ionisation */
#define M3D_GENCOL_CH0 6        /* 'CH0': charge transfer with H-, an upward rate */
#define M3D_GENCOL_UP 7         /* 'UP' + a collider's name: an upward rate */
#define M3D_GENCOL_DN 8         /* 'DN' + a collider's name: a downward rate */

/* The tabulated collision records of an atom file (coll_type, atom_mod.f90:180-191,
 * read at :1412-1530): ln of the rate coefficient at the temperature nodes, which
 * gencol (:2223-2360) interpolates in T by cubic Hermite.  FOSC records fill col_fac
 * instead and are not records here. */
typedef struct m3d_gencol {
  int nrec, ntemp;             /* records, temperature nodes (>= 2) */
  const double *tgrid;         /* (ntemp) ascending [K] */
  const double *lnc;           /* (nrec, ntemp): lnc[rec*ntemp + k], ln of the table values */
  const double *dlnc;          /* same layout: node slopes, or NULL for hermite_derivative's (pchip_slopes8) */
  const int *ll, *ul;          /* (nrec) lower and upper level of the record */
  const int *kind;             /* (nrec) M3D_GENCOL_* */
  const int *collider;         /* (nrec) row of m3d_col_cells_t.colliders for UP/DN, or NULL */
  int ch0_hmip, pad;           /* CH0 rates times exp(-0.754 eV / kT) */
} m3d_gencol_t;

/* The model atom (atom_type, atom_mod.f90:120-160).  Transitions 0..nline-1 are the
 * lines, nline..nrad-1 the continua.  Collision pairs are the (i < j) pairs that
 * classic_col fills with a recipe, each pair at most once: col_kind its electron
 * recipe (0 none), col_hkind its hydrogen one (NULL or 0 none).  gencol adds the
 * atom file's records after them. */
typedef struct m3d_atom {
  int nlevel;                  /* 1..64 */
  int nrad, nline;             /* transitions, of which lines */
  int ncol;                    /* classic_col pairs */
  const int *trans_i, *trans_j;   /* (nrad) lower, upper level */
  const unsigned char *active;    /* (nrad) trans%active, or NULL for all */
  const double *Aji;              /* (nrad) line Einstein A [1/s]; the cut rate of a line */
  const double *g, *ev;           /* (nlevel) statistical weight, energy [eV] */
  const int *ion;                 /* (nlevel) ion stage, 1 = neutral */
  const int *col_i, *col_j, *col_kind; /* (ncol) pair and M3D_COL_* */
  const float *col_fac;           /* (ncol) cdata(tri): f of a line, alpha0 of a continuum, 0 */
  double fmin;                    /* atom_params fmin, (double)1e-6f */
  double cbbesc, cbfesc, colscale, upsilon_floor; /* 1, 1, 1, 0 */
  double cut_x, bf_cut_rate;      /* radiative cut, 70 and 1 [1/s] (atom_mod.f90:256-257) */
  const int *col_hkind;           /* (ncol) M3D_COLH_*, or NULL for electron recipes only */
  double drawin;                  /* prepare_Drawin's prefactor for the atom's weight (atom_mod.f90:1741-1750) */
  double cbbhsc, cbfhsc;          /* factors on the bound-bound and bound-free hydrogen rates, 1 and 1 */
  const m3d_gencol_t *gencol;     /* the atom file's collision records, or NULL */
} m3d_atom_t;

/* The per-cell inputs of the collision rates (collision_rates, atom_mod.f90:918-930),
 * each (ncell) unless stated.  A pointer the atom's recipes do not read may be NULL. */
typedef struct m3d_col_cells {
  const double *temp;          /* [K]; also the tmax_update filter of m3d_stateq_update */
  const double *ne;            /* electron density */
  const double *dxi;           /* ionisation-energy lowering [eV], or NULL for 0 */
  const double *nh1;           /* neutral hydrogen ground level: hydrogen recipes, CH, CHI, CH0 */
  const double *lsaha;         /* comp%lsaha: gencol's n_ul/n_ll where n*_ll = 0 */
  const double *colliders;     /* (ncollider, ncell): the colliders of UP/DN records */
  int ncollider, pad;
} m3d_col_cells_t;

/* Rows of a cup buffer for the atom: ncol electron rates, ncol hydrogen rates with
 * col_hkind, then 2 nrec for gencol's records (upward, then downward). */
int m3d_collision_nrows(const m3d_atom_t *atom);

typedef struct m3d_se_params {
  double max_update;     /* 100 */
  double sor_w;          /* 1 */
  double min_pop_frac;   /* 1e-30 */
  double conv_pop_floor; /* 0 */
  double tmax_update;    /* 1e7 K; needs temp */
  double cswitch;        /* factor on the collision matrix, 0 leaves collisions out */
  int solver;            /* M3D_SE_* */
  int pad;
} m3d_se_params_t;

typedef struct m3d_se_result {
  double maxerr;         /* adata%maxerr: signed largest (conv_pop_floor-weighted) relative change */
  long long epos_cell;   /* its cell, -1 if nothing changed */
  int epos_level;        /* its level, -1 if nothing changed */
  int pad;
  long long nclamp, ntot; /* corrections cut by the limiter, all corrections (ng_count_clamped) */
  long long nonfinite_cell; /* first cell whose solution was not finite, -1 if none */
} m3d_se_result_t;

/* collision_rates (atom_mod.f90:918-930) of every cell: cup (ncell, m3d_collision_nrows)
 * [1/s], colscale applied.  Rows 0..ncol-1 the upward electron rates of classic_col
 * (:1758-1850), then with col_hkind ncol rows of its hydrogen rates (:1854-1876), the
 * downward rate of each being cup * n*_i/n*_j; then with gencol nrec rows of each
 * record's upward and nrec of its downward rate (:2223-2360), for which nstar
 * (ncell, nlevel) is read. */
int m3d_collision_rates(const m3d_atom_t *atom, int ncell, const double *e_kT, const double *nstar,
                        const m3d_col_cells_t *cells, double *cup, unsigned flags);

/* update_populations (atom_mod.f90:439-732) with setup_transition_matrix (:740-841):
 * for every cell with totn > 0 (and temp < tmax_update when cells->temp is given) the
 * rate matrix from gamma_ij/gamma_ji (ncell, nrad) float32 -- a line's thermal and
 * deviation integrals, a continuum's upward and downward rates -- plus
 * collisions x cswitch, the solve, the limiter, e^sor_w, renormalisation to totn and
 * the population floor; b (ncell, nlevel) is updated in place.  Collisions come from
 * cup (as m3d_collision_rates lays it out) when given, else from cells as
 * m3d_collision_rates forms them.  cells may be NULL without collisions or temp
 * filter.  lvlerr (nlevel, host) and res (host) receive the convergence record.
 * A cell whose solution is not finite keeps its b, and the call returns
 * M3D_ENONFINITE with res->nonfinite_cell set (the reference stops the run there).
 * Each cell is solved by a team of threads sharing its matrix: one warp, or for
 * lineq_no_pivot a block of 64 or 128 threads when that keeps more threads resident
 * (large atoms); every element takes the same operations in the same order either
 * way.  M3D_SE_WARP keeps one warp per cell. */
int m3d_stateq_update(const m3d_atom_t *atom, const m3d_se_params_t *par, int ncell, double *b,
                      const double *nstar, const double *totn, const double *e_kT,
                      const m3d_col_cells_t *cells, const float *gamma_ij, const float *gamma_ji,
                      const double *cup, double *lvlerr, m3d_se_result_t *res, unsigned flags);

/* Threads per cell of this thread context's last m3d_stateq_update (32, 64 or 128;
 * 0 before the first).  Diagnostic. */
int m3d_stateq_team(void);

/* ng_accumulate (ng_mod.f90:241-287): gram (host, 7) = d01, d02, d11, d12, d21, d22
 * and |d0|^2 over all cells and levels of ln b; oldb is (ncell, nlevel, 3), the
 * iterates n1, n2, n3. */
int m3d_ng_accumulate(int ncell, int nlevel, const double *b, const double *oldb, double *gram,
                      unsigned flags);

/* ng_extrapolate (ng_mod.f90:314-390): b = exp((1-a-bc) n4 + a n3 + bc n2), renormalised
 * per cell to totn, unless some level would move by more than max_change (or a, bc
 * are not finite): then b is untouched and *applied = 0.  emax, epos_cell, epos_level
 * (host) give the largest relative change. */
int m3d_ng_extrapolate(int ncell, int nlevel, double *b, const double *oldb, const double *nstar,
                       const double *totn, double a, double bc, double max_change, int *applied,
                       double *emax, long long *epos_cell, int *epos_level, unsigned flags);

/* ---- model-atom opacities and ALI rate integrals of one frequency window ----
 * The transitions of the atom in the window (atom_trans_t, hydrogen lines
 * excluded), 0-based.  A line's points f = blue..red of the window (0-based, within
 * 0..nf-1) sit at q[off + f - blue] (likewise wnu, wq); a continuum's at
 * alpha[off + f - blue].  Kinds follow the reference's declarations
 * (trans_mod.f90:20-80, bbtrans_mod.f90:15-25): q and alpha real(4), the rest real(8).
 * The window tables are host memory whatever the flags. */
typedef struct m3d_atom_window {
  int nf, nline, ncont, nlevel;
  const int *line_i, *line_j;       /* (nline) levels */
  const int *line_ntrans;           /* (nline) transition index in the atom: gamma, wphi, psi flag bit */
  const int *line_index;            /* (nline) contribution index of the split tracking, >= 1 */
  const int *line_blue, *line_red, *line_off;
  const float *q;                   /* per line point: 1 - lam/lam0 [Doppler units of idf] */
  const double *wnu, *wq;           /* per line point: rate and profile quadrature weights */
  const double *Bij, *Aij, *lower_ev;       /* (nline) */
  const unsigned char *line_active;         /* (nline) or NULL */
  const unsigned char *sums_over_windows;   /* (nline) */
  const double *grad, *gw1, *gw2, *gstk;    /* (nline) damping constants */
  const unsigned char *unsold;              /* (nline) */
  const int *cont_i, *cont_j, *cont_ntrans, *cont_blue, *cont_red, *cont_off;
  const float *alpha;               /* per continuum point [cm^2] */
  const double *cwnu;               /* per continuum point */
  const unsigned char *cont_active; /* (ncont) or NULL */
  const double *g, *ev;             /* (nlevel) */
  double cut_x;                     /* 70 */
} m3d_atom_window_t;

/* bound_bound_damping (rt_patch_mod.f90:2649-2681): adamp (ncell, nline) */
int m3d_bb_damping(const m3d_atom_window_t *w, int ncell, const float *ne, const float *tothi,
                   const float *vbar2, const float *stark_pe, const float *unsold, const float *inv_df,
                   float *adamp, unsigned flags);

/* add_bound_free_opacities (rt_patch_mod.f90:2581-2643): xhat, ehat (nf, ncell) += ;
 * b (ncell, nlevel) NULL for b = 1; nstar (ncell, nlevel) and pop_ratio, e_kT (ncell)
 * float64 */
int m3d_bf_opacity(const m3d_atom_window_t *w, int ncell, const double *b, const double *nstar,
                   const double *pop_ratio, const double *e_kT, float *xhat, float *ehat,
                   unsigned flags);

/* add_bound_bound_opacities for one direction (rt_patch_mod.f90:2689-2831) into
 * work(:, :, 1:2) = (xhat, ehat), (nf, ncell) each.  With split arrays (all six
 * non-NULL, (nf, ncell)) the tracking starts from (ehat, xhat) as foreground does
 * (:1474-1487) and takes every line's contribution through add_largest.  wphi
 * (ncell, nline of the atom, indexed by line_ntrans) or NULL: the direction's profile
 * integral times wmu is added for the lines that sum over windows (iteration 0). */
int m3d_bb_opacity(const m3d_atom_window_t *w, int ncell, const double *b, const double *nstar,
                   const double *pop_ratio, const double *e_kT, const float *inv_df,
                   const float *vproj, const float *adamp, int lte, float wmu, float *xhat,
                   float *ehat, float *split_opac_L, float *split_opac_R, int *split_id,
                   float *split_chi_L, float *split_chi_R, int *split_chi_id, float *wphi,
                   unsigned flags);

/* m3d_bb_opacity (non-LTE, with the split tracking) and
 * m3d_work_to_transfer_units_split (no scattering term, masers floored) of one
 * direction in one pass, as rt_patch_t%execute runs them back to back: the
 * background xhat, ehat (nf, ncell) is read, the lines added, and every point leaves as
 * chi, S (nf, ncell) with its split arrays.  Equal bit for bit to the two calls on a
 * copy of the background; no count of the floored points. */
int m3d_bb_opacity_units(const m3d_atom_window_t *w, int ncell, const double *b, const double *nstar,
                         const double *pop_ratio, const double *e_kT, const float *inv_df, const float *vproj,
                         const float *adamp, float wmu, const float *xhat, const float *ehat, const float *beta,
                         double maser_chi_floor, float *chi, float *S, float *split_opac_L, float *split_opac_R,
                         int *split_id, float *split_chi_L, float *split_chi_R, int *split_chi_id, float *wphi,
                         unsigned flags);

/* work_to_transfer_units with split rates (rt_patch_mod.f90:3591-3604, 3614-3632):
 * scat = chi_scat*dJnu (nf, ncell) or NULL */
int m3d_work_to_transfer_units_split(int nf, int ncell, float *w1, float *w2, const float *beta,
                                     const float *split_opac_L, const float *split_opac_R,
                                     const float *scat, double maser_chi_floor, int suppress_masers,
                                     int *n_floored, unsigned flags);

/* bound_bound_rates for one direction (rt_patch_mod.f90:2852-3142); gamma_ij/ji
 * (ncell, nline + ncont) of the window, accumulated.  work1 = chi after
 * work_to_transfer_units; inu = work(:,:,3); psi, irem, escape from the formal solver
 * (M3D_GET_PSI, M3D_SPLIT_RATES); the split arrays of m3d_bb_opacity.  psi_flags
 * (ncell, nwords) uint32, bit ntrans%32 of word ntrans/32: flags_in the pairs in
 * force, flags_raise receives the raised ones (atom_data_t psi_flags(:,:,:,:,1:2)). */
typedef struct m3d_rate_opts {
  int split_rates;    /* rate_formulation = 'largest' */
  int preconditioning;
  int per_direction;  /* .not. (do_full_sp .and. fixed_Jnu > 0) */
  int use_flags;
  int do_scat;        /* line scattering: scat given */
  int nwords;
  float wmu, wtot;    /* the direction's weight and the sum of all directions' weights */
} m3d_rate_opts_t;

int m3d_bb_rates(const m3d_atom_window_t *w, const m3d_rate_opts_t *o, int ncell, const double *b,
                 const double *nstar, const double *pop_ratio, const double *e_kT,
                 const float *inv_df, const float *vproj, const float *adamp, const float *work1,
                 const float *inu, const float *psi, const float *irem, const float *escape,
                 const float *beta, const float *Bnu, const float *split_opac_L,
                 const float *split_opac_R, const int *split_id, const float *split_chi_L,
                 const float *split_chi_R, const int *split_chi_id, const float *scat,
                 const unsigned *flags_in, unsigned *flags_raise, float *gamma_ij, float *gamma_ji,
                 unsigned flags);

/* bound_free_rates (rt_patch_mod.f90:3193-3259) from the angle-integrated Jnu and
 * PsiJ (nf, ncell); twohnu3_c2 (nf) */
int m3d_bf_rates(const m3d_atom_window_t *w, int ncell, int preconditioning, const double *b,
                 const double *nstar, const double *e_kT, const float *twohnu3_c2, const float *Jnu,
                 const float *PsiJ, const float *beta, float *gamma_ij, float *gamma_ji,
                 unsigned flags);

/* integrate_rates (rt_patch_mod.f90:3437-3465): the window's (ncell, nline + ncont)
 * sums into the atom's (ncell, nrad) rates by transition index */
int m3d_integrate_rates(const m3d_atom_window_t *w, int ncell, const float *gw_ij, const float *gw_ji,
                        float *gamma_ij, float *gamma_ji, unsigned flags);

/* normalize_profiles (atom_mod.f90:377-430) on the atom's rates (ncell, nrad): in the
 * first iteration wphi -> 1/wphi (1 where wphi = 0); lines with has_wphi scale by
 * wphi; continua scale gamma_ji by n*_i/n*_j.  ti, tj, active, has_wphi host memory. */
int m3d_normalize_profiles(int ncell, int nline, int nrad, const int *ti, const int *tj,
                           const unsigned char *active, const unsigned char *has_wphi,
                           int first_iter, const double *nstar, float *wphi, float *gamma_ij,
                           float *gamma_ji, unsigned flags);

/* combine_twin_hemispheres' average (rt_patch_mod.f90:1812-1887): a = b = (a + b)/2 over n */
int m3d_combine_twins(long long n, float *a, float *b, unsigned flags);

/* ---- inputs and bookkeeping around the solvers ----
 * update_eta_mask (rt_patch_mod.f90:3671-3807) for one slab and set, with the flags
 * kept dense: eta_src and eta_mask (nf, nx, ny, nz), eta_gsrc (nf, nx, ny) of the
 * upstream ghost plane, one byte per point.  work (nf, nx, ny, 0:nz+1, 3) holds
 * (chi, Snu) after work_to_transfer_units and the boundary; beta (nf, nx, ny, nz).
 * rx, ry: the spread eta_rx, eta_ry (floor(max|vx/vz| dz/dx) + 1, 0 for columns);
 * ghost: test the ghost plane (the slab is not at the top of the domain).  The
 * solvers take the dense mask as eta_row(cell) = cell + 1 with eta_mask. */
int m3d_update_eta_mask(const m3d_slab_t *slab, const float *work, const float *beta, unsigned char *eta_src,
                        unsigned char *eta_gsrc, unsigned char *eta_mask, int rx, int ry, int ghost,
                        unsigned flags);

/* compute_lte_populations with the atom's own levels as partition function
 * (level_partf, atom_mod.f90:1041-1140) and lte_pop (:1132-1150): nstar (ncell, nlevel)
 * out, totn (ncell) in (the species' atoms) and out (the sum of nstar).  temp, lsaha =
 * ln(2 (2 pi m_e kT/h^2)^1.5 / ne) and dxi (may be NULL) are float32. */
int m3d_lte_populations(const m3d_atom_t *atom, int ncell, const float *temp, const float *lsaha, const float *dxi,
                        double *nstar, double *totn, unsigned flags);

/* lte_background_emission (rt_patch_mod.f90:2127-2328) with convert_to_work_units
 * (:3518-3536), all (nf, ncell): J is Jnu (jnu_init 0, a later iteration), Bnu (1,
 * initial_Jnu='Planck') or 0 (2, 'zero'); with PsiJ the OAB step of scattering
 * preconditioning, Jali = (J - op Jali_old)/(1 - op), op = sigma PsiJ clamped to
 * [0, scat_op_max], in float64 (Jali in/out, jali_valid 0 seeds it with J; negative
 * results fall back to J and are counted in n_negative); then eta = chi_cont Bnu +
 * sigma (J - Bnu), dJnu = J - Bnu (may be NULL), xhat = chi_cont + eta, ehat = eta/beta.
 * sigma NULL: no continuum scattering.  Jnu itself is not modified. */
int m3d_lte_emission(int nf, int ncell, const float *chi_cont, const float *sigma, const float *Bnu, const float *beta,
                     const float *Jnu, int jnu_init, const float *PsiJ, float *Jali, int jali_valid, double scat_op_max,
                     float *xhat, float *ehat, float *dJnu, long long *n_negative, unsigned flags);

/* add_particle_opacity's per-cell fields of one isotope (linelist_mod.f90:1023-1042,
 * ion_mod.f90:198-221): inv_df, vbar2 and lnbase = ln max(n, tiny) [+ ln scale] - part
 * + ln inv_df + ln iso_frac; n and part (the log partition function) float64.
 * population_scale 0 = none. */
int m3d_particle_fields(int ncell, double awgt, float vmic, double iso_frac, double population_scale,
                        const float *temp, const double *n, const double *part, float *inv_df, float *vbar2,
                        float *lnbase, unsigned flags);

/* ---- batched 1.5D ALI: columns of uneven depth -------------------------------------
 * The cells of all columns lie back to back: column c owns cells col_off[c] ..
 * col_off[c+1]-1, bottom to top, each with its own cell height dz[c] [cm].  The
 * per-cell inputs are device pointers the caller keeps alive for the plan's life
 * (b and nstar (nlevel, ncell) float64; pop_ratio and e_kT (ncell) float64; inv_df,
 * vz [c], chi_c (the grey continuum [1/cm]) and temp (ncell) float32).  mu/wmu are
 * the directions (host): the upward half, then the same mirrored, mean-intensity
 * weights (nphi_copies with Jnu_weights).  bottom: M3D_BND_PCHIP or M3D_BND_ZERO for
 * the ghost of upward rays; downward rays enter through a zero top. */
typedef struct {
  int ncol, ncell;
  const int *col_off;    /* ncol+1 (device) */
  const double *dz;      /* ncol (device) */
  int nray;
  const double *mu;      /* nray (host) */
  const float *wmu;      /* nray (host) */
  const double *b, *nstar, *pop_ratio, *e_kT;
  const float *inv_df, *vz, *chi_c, *temp;
  double maser_dtau_max, maser_Inu_max, maser_chi_floor;
  int preconditioning, bottom;
  int nline_atom, nrad_atom;  /* the atom's lines and transitions (rows of wphi and gamma) */
} m3d_col_problem_t;

typedef struct m3d_col_plan m3d_col_plan_t;

/* A plan for one model atom over its frequency windows: the windows' tables are
 * staged once (win_nu float64, win_twohnu3_c2 float32 per window, host or device;
 * win_adamp the window lines' damping (nline, ncell), device), and the plan owns
 * work arrays sized for the widest window.  A window whose every frequency lies in
 * at most 4 line windows is swept by one fused kernel per hemisphere (line opacity,
 * transfer units, the column solve, J/PsiJ and the line rates of a column in one
 * CTA); the others, and every window with M3D_COL_PERPOINT, by the per-point
 * kernels.  Both give the same bits.  With M3D_AUTOTUNE the launch shapes (the
 * fused kernel's threads per column and cells per chunk, the column solver's block
 * size) are chosen by timing. */
int m3d_col_plan_create(const m3d_col_problem_t *p, int nwin, const m3d_atom_window_t *wins,
                        const double *const *win_nu, const float *const *win_twohnu3_c2,
                        const float *const *win_adamp, unsigned flags, m3d_col_plan_t **plan);
/* One ALI sweep over every window and direction (rt_patch_t%execute's ALI branch
 * for both hemisphere twins, the long characteristics along each column): the
 * rates accumulate into gamma_ij/gamma_ji (nrad_atom, ncell, device) and, with
 * first_iter, the profile integrals into wphi (nline_atom, ncell, device; may be
 * NULL).  The sweep is a fixed sequence of launches on the library stream; with
 * use_graph it is captured once per (first_iter, gamma, wphi) into a CUDA graph and
 * replayed. */
int m3d_col_plan_sweep(m3d_col_plan_t *plan, int first_iter, float *gamma_ij, float *gamma_ji, float *wphi,
                       int use_graph);
/* Copies the combined J and PsiJ of the last window (2 x (ncell, nf): both twins
 * hold the average) into J, PsiJ (host or device, may be NULL) and returns that
 * window's nf and the block size of the sweep's solver (the fused kernel's when
 * every window is fused); synchronises. */
int m3d_col_plan_fields(m3d_col_plan_t *plan, float *J, float *PsiJ, int *nf, int *solver_block);
/* The plan's launch shapes: how many windows the fused kernel sweeps, its threads
 * per column and cells per chunk, the per-point column solver's block size (any
 * pointer may be NULL). */
int m3d_col_plan_shape(m3d_col_plan_t *plan, int *fused_windows, int *fused_block, int *zchunk, int *solver_block);
int m3d_col_plan_destroy(m3d_col_plan_t *plan);

/* Self-check with no counterpart in the reference.  The opacity kernels form 1/(1+u)
 * by one Markstein step from the approximate reciprocal wherever the window bounds
 * 1+u below 2^126, and rely on it being bit-identical to the correctly rounded
 * reciprocal there.  This compares the two on every float whose bit pattern lies in
 * [lo_bits, hi_bits) on the current device: mismatches and the first mismatching
 * pattern (0xffffffff if none) come back on the host. */
int m3d_rcp_check(unsigned lo_bits, unsigned hi_bits, unsigned long long *mismatches, unsigned *first_bits);

#ifdef __cplusplus
}
#endif
#endif /* M3DGPU_H */

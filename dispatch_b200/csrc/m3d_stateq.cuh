// Statistical equilibrium on the device, FP64: the rate matrix of every cell
// (setup_transition_matrix, SRC/atom_mod.f90:740-841, with line_rate_coefficients
// :862-884 and the electron and hydrogen recipes of classic_col :1758-1880), its dense solve
// (lineq_no_pivot / lineq, HOP/op_math_mod.f90:263-356, 420-449, or LU with
// partial pivoting) and the population update (update_populations :439-732);
// then Ng's accumulation and extrapolation in ln b (SRC/ng_mod.f90:241-390).
//
// One warp owns one cell at a time and keeps the cell's rate matrix (column
// major, n <= 64) and its vectors in shared memory.  Every elimination step
// updates each matrix element once, so spreading a step's elements over the
// lanes performs exactly the roundings of the sequential loops; the
// substitutions that a row-wise loop orders differently from a column-wise one
// run column by column where the orders agree and on one lane where they do
// not (the back substitution of lineq_no_pivot).  The library is compiled with
// -fmad=false, so no product is fused into a sum.
#pragma once
#include <cfloat>
#include <cstdint>

namespace m3d {

constexpr int SE_NMAX = 64;
constexpr int SE_COL_REGEMORTER = 1, SE_COL_SEATON = 2;
constexpr int SE_COLH_DRAWIN = 1, SE_COLH_TAKEDA = 2;

// Atom tables in device memory.  Transitions are listed by round: the
// transitions of one round touch pairwise different matrix elements, and a
// pair's transitions fall in successive rounds in their original order, so
// the additions into each element keep the reference's transition order.
struct SeAtomDev {
  int n, nline, nround, ncol;
  const int *order;      // transition index, grouped by round (active ones only)
  const int *round_off;  // [nround + 1]
  const int *ti, *tj;    // [nrad]
  const double *Aji;     // [nrad]
  const double *g, *ev;  // [n]
  const int *ion;        // [n]
  const int *ci, *cj, *ckind;  // [ncol]
  const float *cfac;           // [ncol]
  const int *chkind;           // [ncol] hydrogen recipes, or null: none
  double fmin, cbbesc, cbfesc, colscale, upsilon_floor, cut_x, bf_cut_rate;
  double drawin, cbbhsc, cbfhsc;
  // gencol's records (atom_mod.f90:2223-2360) and, with records, the matrix
  // elements that collisions reach: element e is W[el_w[e]], its contributions
  // el_src[el_off[e] .. el_off[e+1]) in the order the reference adds them, each
  // (index << 2 | type), type 0/1 a classic pair's upward/downward rate, 2/3 a
  // record's upward/downward rate
  int ngrec, ntemp, ch0_hmip, nel;
  const double *gt, *glnc, *gdc;  // [ntemp], [ngrec * ntemp] x 2
  const int *gll, *gul, *gkind, *gcoll;
  const int *el_w, *el_off, *el_src;
};

struct SeParams {
  double max_update, sor_w, min_pop_frac, conv_pop_floor, tmax_update, cswitch;
  int solver;
};

struct SeCells {
  int ncell;
  double *b;
  const double *nstar, *totn, *temp, *ne, *e_kT, *dxi, *nh1, *lsaha, *coll;
  const float *gij, *gji;
  const double *cup;  // precomputed collision rates, or null to form them here
};

// per-warp partial results of the convergence measures
struct SeWarpBest {
  double maxerr_abs, maxerr;  // weighted |e| and the signed value
  long long cell;             // -1: none
  int level, pad;
};

// ---- classic_col helpers (atom_mod.f90:2362-2467) ------------------------------
// The Fortran tables are default-real literals: their single-precision values
// enter the double arithmetic.
__device__ __forceinline__ double se_expin(double x) {
  const float a0 = -44178.5471728217f, a1 = 57721.7247139444f, a2 = 9938.31388962037f, a3 = 1842.11088668000f,
              a4 = 101.093806161906f, a5 = 5.03416184097568f;
  const float b0 = 76537.3323337614f, b1 = 32597.1881290275f, b2 = 6106.10794245759f, b3 = 635.419418378382f,
              b4 = 37.2298352833327f;
  const float c0 = 4.65627107975096e-7f, c1 = .999979577051595f, c2 = 9.04161556946329f, c3 = 24.3784088791317f,
              c4 = 23.0192559391333f, c5 = 6.90522522784444f, c6 = .430967839469389f;
  const float d0 = 10.0411643829054f, d1 = 32.4264210695138f, d2 = 41.2807841891424f, d3 = 20.4494785013794f,
              d4 = 3.31909213593302f, d5 = .103400130404874f;
  const float e0 = -.999999999998447f, e1 = -26.6271060431811f, e2 = -241.055827097015f, e3 = -895.927957772937f,
              e4 = -1298.85688746484f, e5 = -545.374158883133f, e6 = -5.66575206533869f;
  const float f0 = 28.6271060422192f, f1 = 292.310039388533f, f2 = 1332.78537748257f, f3 = 2777.61949509163f,
              f4 = 2404.01713225909f, f5 = 631.657483280800f;
  const double ex = exp(-x);
  if (x > 4) {
    return (ex + ex * ((double)e0 + ((double)e1 + ((double)e2 + ((double)e3 + ((double)e4 + ((double)e5 + (double)e6 / x) / x) / x) / x) / x) / x) /
                     (x + (double)f0 + ((double)f1 + ((double)f2 + ((double)f3 + ((double)f4 + (double)f5 / x) / x) / x) / x) / x)) /
           x;
  } else if (x > 1) {
    return ex * ((double)c6 + ((double)c5 + ((double)c4 + ((double)c3 + ((double)c2 + ((double)c1 + (double)c0 * x) * x) * x) * x) * x) * x) /
           ((double)d5 + ((double)d4 + ((double)d3 + ((double)d2 + ((double)d1 + ((double)d0 + x) * x) * x) * x) * x) * x);
  } else if (x > 0) {
    return ((double)a0 + ((double)a1 + ((double)a2 + ((double)a3 + ((double)a4 + (double)a5 * x) * x) * x) * x) * x) /
               ((double)b0 + ((double)b1 + ((double)b2 + ((double)b3 + ((double)b4 + x) * x) * x) * x) * x) -
           log(x);
  }
  return 0.0;
}

__constant__ float se_gaunt_a1[6] = {1.078e00f, 1.0926e0f, 1.0983e0f, 1.0954e0f, 1.0912e0f, 1.0925e0f};
__constant__ float se_gaunt_b1[6] = {-8.754e14f, -2.019e14f, -9.45e13f, -5.188e13f, -3.2e13f, -2.331e13f};
__constant__ float se_gaunt_c1[6] = {-1.791e29f, 1.836e28f, 9.177e27f, 3.552e27f, 1.576e27f, 9.325e26f};
__constant__ float se_gaunt_a2[6] = {0.798e00f, 0.768e00f, 0.793e00f, 0.831e00f, 0.758e00f, 0.79e00f};
__constant__ float se_gaunt_b2[6] = {5.358e15f, 6.242e15f, 5.48e15f, 4.094e15f, 6.633e15f, 5.808e15f};
__constant__ float se_gaunt_c2[6] = {-3.484e31f, -3.208e31f, -2.318e31f, -1.43e31f, -3.32e31f, -2.844e31f};

__device__ __forceinline__ double se_gaunt(double lam, int n) {
  const float *a1 = se_gaunt_a1, *b1 = se_gaunt_b1, *c1 = se_gaunt_c1;
  const float *a2 = se_gaunt_a2, *b2 = se_gaunt_b2, *c2 = se_gaunt_c2;
  const double inv_nu = lam * (1e-8 / 2.99792458e10);
  if (n > 6) return 1.0;
  if (inv_nu >= (double)1e-16f) return (double)a1[n - 1] + ((double)b1[n - 1] + (double)c1[n - 1] * inv_nu) * inv_nu;
  return (double)a2[n - 1] + ((double)b2[n - 1] + (double)c2[n - 1] * inv_nu) * inv_nu;
}

// Kramers' cross section; kramer_const = 64 PI^4 EC^10 EM / (3 sqrt(3) CC HH^6)
// with each power and product rounded to double once
__device__ __forceinline__ double se_kramer(double lam, double dev) {
  const double nu = (2.99792458e10 / 1e-8) / lam;
  if (dev > 0) {
    const double nl = sqrt(13.605 / dev);
    const double nl2 = nl * nl, nl5 = nl * (nl2 * nl2), nu3 = nu * (nu * nu);
    return 0x1.c6dc1aa1038f0p+97 * se_gaunt(lam, (int)ceil(nl)) / (nl5 * nu3);
  }
  return 0.0;
}

struct SeColCell { double allen, regemorter, seaton, ekt, dxi, sqt, ne, nh1; };

__device__ __forceinline__ SeColCell se_col_cell(double temp, double ne, double ekt, double dxi, double nh1) {
  const double PI = 3.14159265359, BK = 1.380662e-16, EM = 9.109534e-28, RB = 5.29177349e-9;
  const double E_K = 1.602189e-12 / BK, RYDK = 13.605 * E_K;
  const double sq8bmp = sqrt(8 * BK / EM / PI);
  const double c0 = PI * (RB * RB) * sq8bmp;
  const double sqt = sqrt(temp);
  SeColCell w;
  w.allen = c0 * RYDK * ne / sqt;
  w.regemorter = 14.5 * w.allen * RYDK / E_K;
  w.seaton = (double)1.55e13f * ne / sqt;
  w.ekt = ekt;
  w.dxi = dxi;
  w.sqt = sqt;
  w.ne = ne;
  w.nh1 = nh1;
  return w;
}

// upward collision rates of pair p [1/s], colscale applied: ue by the pair's
// electron recipe, uh by its hydrogen recipe (0 without one).  The electron mass
// ame of the hydrogen recipes is a default-real literal (atom_mod.f90:220-222).
template <bool HYD>
__device__ __forceinline__ void se_col_rates(const SeAtomDev &A, const SeColCell &w, int p, double &ue,
                                             double &uh) {
  const double sqr3_2pi = (sqrt(3.0) / 2.0) / 3.14159265359;
  const int i = A.ci[p], j = A.cj[p], kind = A.ckind[p];
  const int ioni = A.ion[i], ionj = A.ion[j];
  const bool cont = ionj > ioni;
  double fac = (double)A.cfac[p], f = 0;
  double dev = A.ev[j] - A.ev[i];
  dev = fmax(dev, 1e-8);
  if (cont) {
    const int jj = ionj * (ionj - 1), ii = ioni * (ioni - 1);
    dev = dev - w.dxi * 0.5 * (double)(jj - ii);
  } else {
    f = fmax(fac, A.fmin * A.g[j]);
  }
  const double u0 = dev * w.ekt;
  const double ex = exp(-u0);
  double v = 0;
  if (cont && kind == SE_COL_SEATON) {
    if (fac == 0) {
      const double lam0 = (2.99792458e10 / 1e-8) * (6.626176e-27 / 1.602189e-12) / dev;
      fac = se_kramer(lam0, dev);
    }
    const double tmp = (double)fminf(0.1f * (float)ioni, 0.3f);
    v = w.seaton * fac * tmp / u0 * ex;
    v = v * A.cbfesc;
  } else if (!cont && kind == SE_COL_REGEMORTER) {
    const double tmp = fmax((double)0.2f * ex, sqr3_2pi * se_expin(u0));
    v = w.regemorter * f * tmp / dev;
    v = fmax(v, w.allen * A.upsilon_floor * ex / A.g[i]);
    v = v * A.cbbesc;
  }
  if (v != 0) v = v * A.colscale;
  ue = v;
  uh = 0;
  if (!HYD) return;
  // hydrogen (atom_mod.f90:1854-1876): Takeda for a line without an f value,
  // else Drawin
  const int hkind = A.chkind ? A.chkind[p] : 0;
  double h = 0;
  const double ame = (double)5.485799e-4f, amh = 1.0;
  if (!cont && (double)A.cfac[p] == 0 && hkind == SE_COLH_TAKEDA) {
    h = w.nh1 * (w.allen / w.ne) * (double)ioni / A.g[i] * ex * sqrt(ame / amh);
    h = h * A.cbbhsc;
  } else if (hkind == SE_COLH_DRAWIN) {
    const double mu_e = ame / (ame + amh);
    const double q = 13.605 / dev;
    const double divu = q * q;
    double tmp = 2.0 / u0;
    const double mt = mu_e * tmp;
    tmp = (1.0 + tmp) / (1.0 + mt * mt);
    h = w.nh1 * A.drawin * divu * tmp * ex * w.sqt;
    if (cont) {
      h = h * A.cbfhsc;
    } else {
      h = h * f;
      h = h * A.cbbhsc;
    }
  }
  if (h != 0) h = h * A.colscale;
  uh = h;
}

// ---- gencol (atom_mod.f90:2223-2360) -------------------------------------------
// hermite_interpolation_single (interpol_mod.f90:558-578): the end values outside
// the nodes, else BinarySearch8's bracket (op_math_mod.f90:179-199), x[i] < xx <=
// x[i+1], and hermite_value8 (interpol_mod.f90:149-162)
__device__ __forceinline__ double se_hermite8(const double *x, const double *y, const double *m, int n,
                                              double xx) {
  if (xx <= x[0]) return y[0];
  if (xx >= x[n - 1]) return y[n - 1];
  int l = 0, r = n - 1;
  while (r - l > 1) {
    const int mid = l + (r - l) / 2;
    if (x[mid] >= xx) r = mid;
    else l = mid;
  }
  const double h = x[l + 1] - x[l];
  const double t = (xx - x[l]) / h;
  const double t2 = t * t, t3 = t2 * t;
  const double p = 3.0 * t2 - 2.0 * t3;
  return (1.0 - p) * y[l] + p * y[l + 1] + h * ((t3 - 2.0 * t2 + t) * m[l] + (t3 - t2) * m[l + 1]);
}

// record r's upward and downward rates [1/s], colscale applied; nll, nul the
// cell's n* of the record's levels, ncoll its collider's density (UP/DN)
__device__ __forceinline__ void se_gencol_rates(const SeAtomDev &A, int r, double temp, double ne, double dxi,
                                                double nh1, double lsaha, double ncoll, double ekt, double nll,
                                                double nul, double &up, double &dn) {
  const double PI = 3.14159265359, BK = 1.380662e-16, EM = 9.109534e-28, RB = 5.29177349e-9;
  const double ERYD = 13.605 * 1.602189e-12;
  const double c0 = ((ERYD / sqrt(EM)) * PI * (RB * RB)) * sqrt(8.0 / (PI * BK));
  const int ll = A.gll[r], ul = A.gul[r], kind = A.gkind[r];
  double dev = A.ev[ul] - A.ev[ll];
  if (A.ion[ul] > A.ion[ll]) {
    const int ii = A.ion[ll] * (A.ion[ll] - 1), jj = A.ion[ul] * (A.ion[ul] - 1);
    dev = dev - dxi * 0.5 * (double)(jj - ii);
  }
  double nji;
  if (nll > 0) {
    nji = nul / nll;
  } else {
    const double tns = -(dev * ekt) + (double)(A.ion[ul] - A.ion[ll]) * lsaha;
    nji = A.g[ul] / A.g[ll] * exp(tns);
  }
  const double stg = sqrt(temp);
  const size_t o = (size_t)r * A.ntemp;
  const double ct = exp(se_hermite8(A.gt, A.glnc + o, A.gdc + o, A.ntemp, temp));
  double u = 0, d = 0;
  switch (kind) {
    case 1:  // OHM
      d = c0 / A.g[ul] * ct * ne / stg;
      u = d * nji;
      break;
    case 2:  // CE
      d = A.g[ll] / A.g[ul] * ct * ne * stg;
      d = d * A.cbbesc;
      u = d * nji;
      break;
    case 3:  // CH
      d = ct * nh1;
      d = d * A.cbbhsc;
      u = d * nji;
      break;
    case 4:  // CHI
      u = ct * nh1;
      u = u * A.cbfhsc;
      d = u / nji;
      break;
    case 5:  // CI
      u = ct * ne * stg * exp(-(A.ev[ul] - A.ev[ll]) * ekt);
      u = u * A.cbfesc;
      d = u / nji;
      break;
    case 6:  // CH0; 0.754 is a default-real literal
      u = ct * nh1;
      if (A.ch0_hmip) u = u * exp(-(double)0.754f * ekt);
      u = u * A.cbfhsc;
      d = u / nji;
      break;
    case 7:  // UP
      u = ct * ncoll;
      d = u / nji;
      break;
    case 8:  // DN
      d = ct * ncoll;
      u = d * nji;
      break;
    default:
      break;
  }
  up = u * A.colscale;
  dn = d * A.colscale;
}

// cup[cell + ncell*p] the electron rates; with hydrogen recipes
// cup[cell + ncell*(ncol + p)] the hydrogen ones.  One thread per cell.
// cup[cell + ncell*(r0 + r)] and cup[cell + ncell*(r0 + ngrec + r)] record r's
// upward and downward rates, r0 = ncol (x2 with hydrogen recipes).
__global__ void k_collision_rates(SeAtomDev A, SeCells C, double *__restrict__ cup) {
  const int ncell = C.ncell;
  const int r0 = A.chkind ? 2 * A.ncol : A.ncol;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
    const double dxi = C.dxi ? C.dxi[c] : 0.0, nh1 = C.nh1 ? C.nh1[c] : 0.0;
    const SeColCell w = se_col_cell(C.temp[c], C.ne[c], C.e_kT[c], dxi, nh1);
    for (int p = 0; p < A.ncol; p++) {
      double ue, uh;
      se_col_rates<true>(A, w, p, ue, uh);
      cup[(size_t)c + (size_t)ncell * p] = ue;
      if (A.chkind) cup[(size_t)c + (size_t)ncell * (A.ncol + p)] = uh;
    }
    for (int r = 0; r < A.ngrec; r++) {
      const int k = A.gcoll ? A.gcoll[r] : -1;
      const double nc = k >= 0 ? C.coll[(size_t)c + (size_t)ncell * k] : 0.0;
      double up, dn;
      se_gencol_rates(A, r, C.temp[c], C.ne[c], dxi, nh1, C.lsaha ? C.lsaha[c] : 0.0, nc, C.e_kT[c],
                      C.nstar[(size_t)c + (size_t)ncell * A.gll[r]], C.nstar[(size_t)c + (size_t)ncell * A.gul[r]],
                      up, dn);
      cup[(size_t)c + (size_t)ncell * (r0 + r)] = up;
      cup[(size_t)c + (size_t)ncell * (r0 + A.ngrec + r)] = dn;
    }
  }
}

// ---- the per-warp dense solvers ------------------------------------------------
// a(i,j) = W[i + n*j]; e is the right-hand side, the solution on return.

// A cell's team: TEAM threads share its matrix, one warp (TEAM = 32) or a whole
// block of 64 or 128 threads, whose barriers are then the block's.
template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if (TEAM == 32) __syncwarp();
  else __syncthreads();
}

template <int TEAM>
__device__ __forceinline__ bool team_all(bool v) {
  if (TEAM == 32) return __all_sync(0xffffffffu, v);
  return __syncthreads_and(v) != 0;
}

// a(i,j) - l a(k,j) of one element; SKIP: left alone where a(k,j) = 0, as
// lineq_no_pivot skips it
template <bool SKIP>
__device__ __forceinline__ double se_elim(double aij, double l, double akj) {
  if (SKIP) return akj != 0 ? aij - l * akj : aij;
  return aij - l * akj;
}

// One elimination step k: the multipliers l(i) = a(i,k)/a(k,k) of the rows below
// k go to lstore[i] (column k of W itself, or a separate vector), and the trailing
// block takes a(i,j) - l(i) a(k,j).  A lane owns the rows k+1+lane (and k+33+lane
// while more than 32 rows remain); when fewer rows than lanes remain, the lanes split
// the columns into G groups.  l(i) stays in a register and four columns' loads
// precede their stores, so the FP64 chains of a lane overlap.  Every element takes
// its one update per step, so the roundings are the sequential loop's.
template <bool SKIP, int TEAM = 32>
__device__ __forceinline__ void se_elim_step(double *W, double *lstore, int n, int k, int lane) {
  const int m = n - k - 1;
  const double pk = W[k + n * k];
  const int G = m >= TEAM ? 1 : TEAM / m;
  const int g = m >= TEAM ? 0 : lane / m;
  const bool act = g < G;
  const int i0 = k + 1 + (m >= TEAM ? lane : lane % m), i1 = i0 + TEAM;
  const bool two = m > TEAM && i1 < n;
  double l0 = 0, l1 = 0;
  if (act) {
    l0 = W[i0 + n * k] / pk;
    if (two) l1 = W[i1 + n * k] / pk;
  }
  team_sync<TEAM>();  // every group has read a(i,k) before group 0 may overwrite it with l(i)
  if (act) {
    if (g == 0) {
      lstore[i0] = l0;
      if (two) lstore[i1] = l1;
    }
    int j = k + 1 + g;
    for (; j + 3 * G < n; j += 4 * G) {
      const int c0 = n * j, c1 = c0 + n * G, c2 = c1 + n * G, c3 = c2 + n * G;
      const double a0 = W[k + c0], a1 = W[k + c1], a2 = W[k + c2], a3 = W[k + c3];
      const double x0 = W[i0 + c0], x1 = W[i0 + c1], x2 = W[i0 + c2], x3 = W[i0 + c3];
      if (two) {
        const double y0 = W[i1 + c0], y1 = W[i1 + c1], y2 = W[i1 + c2], y3 = W[i1 + c3];
        W[i1 + c0] = se_elim<SKIP>(y0, l1, a0);
        W[i1 + c1] = se_elim<SKIP>(y1, l1, a1);
        W[i1 + c2] = se_elim<SKIP>(y2, l1, a2);
        W[i1 + c3] = se_elim<SKIP>(y3, l1, a3);
      }
      W[i0 + c0] = se_elim<SKIP>(x0, l0, a0);
      W[i0 + c1] = se_elim<SKIP>(x1, l0, a1);
      W[i0 + c2] = se_elim<SKIP>(x2, l0, a2);
      W[i0 + c3] = se_elim<SKIP>(x3, l0, a3);
    }
    for (; j < n; j += G) {
      const double a = W[k + n * j];
      if (two) W[i1 + n * j] = se_elim<SKIP>(W[i1 + n * j], l1, a);
      W[i0 + n * j] = se_elim<SKIP>(W[i0 + n * j], l0, a);
    }
  }
  team_sync<TEAM>();
}

// lineq_no_pivot (op_math_mod.f90:420-449)
template <int TEAM = 32>
__device__ __forceinline__ void se_solve_no_pivot(double *W, double *e, int n, int lane) {
  for (int k = 0; k < n - 1; k++) se_elim_step<true, TEAM>(W, W + n * k, n, k, lane);
  // forward substitution: per row the terms arrive in ascending j, as in the row loop
  for (int j = 0; j < n - 1; j++) {
    const double ej = e[j];
    for (int i = j + 1 + lane; i < n; i += TEAM) e[i] = e[i] - W[i + n * j] * ej;
    team_sync<TEAM>();
  }
  // back substitution: the row loop adds its terms in ascending j, an order no
  // column sweep reproduces, so one lane runs it
  if (lane == 0) {
    for (int i = n - 1; i >= 0; i--) {
      double t = e[i];
      for (int j = i + 1; j < n; j++) t = t - W[i + n * j] * e[j];
      e[i] = t / W[i + n * i];
    }
  }
  team_sync<TEAM>();
}

// warp arg-max: largest v, ties to the smallest idx; idx < 0 never wins
__device__ __forceinline__ void warp_argmax(double &v, int &idx) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    const bool take = oi >= 0 && (idx < 0 || ov > v || (ov == v && oi < idx));
    if (take) { v = ov; idx = oi; }
  }
}

// the team's arg-max: warp_argmax in each warp, then the warps' winners in warp
// order with the same rule (largest v, ties to the smallest idx); every thread
// returns the result
template <int TEAM>
__device__ __forceinline__ void team_argmax(double &v, int &idx) {
  warp_argmax(v, idx);
  if (TEAM == 32) return;
  constexpr int NW = TEAM / 32 > 0 ? TEAM / 32 : 1;
  __shared__ double tv[NW];
  __shared__ int ti[NW];
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    tv[threadIdx.x >> 5] = v;
    ti[threadIdx.x >> 5] = idx;
  }
  __syncthreads();
  double bv = tv[0];
  int bi = ti[0];
  for (int w = 1; w < NW; w++) {
    const double ov = tv[w];
    const int oi = ti[w];
    if (oi >= 0 && (bi < 0 || ov > bv || (ov == bv && oi < bi))) {
      bv = ov;
      bi = oi;
    }
  }
  v = bv;
  idx = bi;
}

// lineq: Gaussian elimination with full pivoting (op_math_mod.f90:263-356)
__device__ __forceinline__ void se_solve_lineq(double *W, double *e, double *q, int *icol, int n, int lane) {
  for (int i = lane; i < n; i += 32) icol[i] = i;
  __syncwarp();
  for (int s = 0; s < n - 1; s++) {
    // pivot: the first element in row-major order of the largest |a|; the
    // sequential scan starts from |a(s,s)| and moves only on a strict increase
    const int m = n - s;
    double bv = -1.0;
    int bi = -1;
    for (int idx = lane; idx < m * m; idx += 32) {
      const int i = s + idx / m, j = s + idx % m;
      const double a = fabs(W[i + n * j]);
      const double v = a == a ? a : INFINITY;  // a NaN pivot, taken alike by every lane
      if (bi < 0 || v > bv) { bv = v; bi = idx; }
    }
    warp_argmax(bv, bi);
    const int ima = s + bi / m, jma = s + bi % m;
    for (int i = lane; i < n; i += 32) {
      const double t = W[i + n * jma];
      W[i + n * jma] = W[i + n * s];
      W[i + n * s] = t;
    }
    __syncwarp();
    for (int j = s + lane; j < n; j += 32) {
      const double t = W[ima + n * j];
      W[ima + n * j] = W[s + n * j];
      W[s + n * j] = t;
    }
    if (lane == 0) {
      const double t = e[ima];
      e[ima] = e[s];
      e[s] = t;
      const int it = icol[s];
      icol[s] = icol[jma];
      icol[jma] = it;
    }
    __syncwarp();
    se_elim_step<false>(W, q, n, s, lane);
    const double es = e[s];
    for (int i = s + 1 + lane; i < n; i += 32) e[i] = e[i] - q[i] * es;
    __syncwarp();
  }
  // back substitution: the row loop runs j downwards, as a column sweep does
  if (lane == 0) e[n - 1] = e[n - 1] / W[(n - 1) + n * (n - 1)];
  __syncwarp();
  for (int j = n - 1; j >= 1; j--) {
    const double ej = e[j];
    for (int i = lane; i < j; i += 32) e[i] = e[i] - W[i + n * j] * ej;
    __syncwarp();
    if (lane == 0) e[j - 1] = e[j - 1] / W[(j - 1) + n * (j - 1)];
    __syncwarp();
  }
  // reorder: c(icol(i)) = b(i)
  for (int i = lane; i < n; i += 32) q[icol[i]] = e[i];
  __syncwarp();
  for (int i = lane; i < n; i += 32) e[i] = q[i];
  __syncwarp();
}

// LU with partial (row) pivoting: pivot of column k the first row of largest
// |a(i,k)|, i >= k; forward substitution by columns ascending, back
// substitution by columns descending
__device__ __forceinline__ void se_solve_partial(double *W, double *e, int n, int lane) {
  for (int k = 0; k < n - 1; k++) {
    double bv = -1.0;
    int bi = -1;
    for (int i = k + lane; i < n; i += 32) {
      const double a = fabs(W[i + n * k]);
      const double v = a == a ? a : INFINITY;
      if (bi < 0 || v > bv) { bv = v; bi = i; }
    }
    warp_argmax(bv, bi);
    const int p = bi;
    if (p != k) {
      for (int j = lane; j < n; j += 32) {
        const double t = W[k + n * j];
        W[k + n * j] = W[p + n * j];
        W[p + n * j] = t;
      }
      if (lane == 0) {
        const double t = e[k];
        e[k] = e[p];
        e[p] = t;
      }
    }
    __syncwarp();
    se_elim_step<false>(W, W + n * k, n, k, lane);
  }
  for (int j = 0; j < n - 1; j++) {
    const double ej = e[j];
    for (int i = j + 1 + lane; i < n; i += 32) e[i] = e[i] - W[i + n * j] * ej;
    __syncwarp();
  }
  for (int j = n - 1; j >= 0; j--) {
    if (lane == 0) e[j] = e[j] / W[j + n * j];
    __syncwarp();
    const double ej = e[j];
    for (int i = lane; i < j; i += 32) e[i] = e[i] - W[i + n * j] * ej;
    __syncwarp();
  }
}

// shared memory of one warp, in doubles (plus n ints for lineq's column order)
__host__ __device__ inline size_t se_warp_doubles(int n) { return (size_t)n * n + 4 * (size_t)n + (size_t)(n + 1) / 2; }

// update_populations over all cells: warps stride over the cells in ascending order
// CM 0: collision rates read from C.cup (or none); 1: formed here, electron
// recipes only; 2: formed here, any recipes and records.  The host picks the
// least general form, which keeps the common ones' register use down.
template <int CM, int TEAM = 32>
__global__ void k_stateq_update(SeAtomDev A, SeParams P, SeCells C, SeWarpBest *__restrict__ wbest,
                                double *__restrict__ lvl_val, long long *__restrict__ lvl_cell,
                                unsigned long long *__restrict__ counts, long long *__restrict__ nonfinite) {
  extern __shared__ double se_smem[];
  // a team of TEAM threads per cell: a warp (several teams per block), or the block
  const int n = A.n, lane = TEAM == 32 ? (int)(threadIdx.x & 31) : (int)threadIdx.x;
  const int wib = TEAM == 32 ? (int)(threadIdx.x >> 5) : 0;
  double *W = se_smem + se_warp_doubles(n) * wib;
  double *bl = W + n * n, *ns = bl + n, *e = ns + n, *q = e + n;
  int *icol = (int *)(q + n);
  const int tpb = TEAM == 32 ? (int)(blockDim.x >> 5) : 1;  // teams per block
  const int nwarp = gridDim.x * tpb;
  const int gw = blockIdx.x * tpb + wib;
  const int ncell = C.ncell;
  const double eup = fmax(P.max_update, 1.0), elo = 1.0 / eup;

  SeWarpBest best;
  best.maxerr_abs = 0;
  best.maxerr = 0;
  best.cell = -1;
  best.level = -1;
  best.pad = 0;
  double lv[2] = {0, 0};
  long long lc[2] = {-1, -1};
  unsigned long long nclamp = 0, ntot = 0;

  for (int c = gw; c < ncell; c += nwarp) {
    const double totn = C.totn[c];
    if (!(totn > 0)) continue;
    if (C.temp && !(C.temp[c] < P.tmax_update)) continue;
    const double ekt = C.e_kT[c];
    for (int k = lane; k < n; k += TEAM) {
      bl[k] = C.b[(size_t)c + (size_t)ncell * k];
      ns[k] = C.nstar[(size_t)c + (size_t)ncell * k];
      e[k] = 0;
    }
    for (int idx = lane; idx < n * n; idx += TEAM) W[idx] = 0;
    team_sync<TEAM>();
    // radiative rates, round by round
    for (int r = 0; r < A.nround; r++) {
      for (int t = A.round_off[r] + lane; t < A.round_off[r + 1]; t += TEAM) {
        const int kr = A.order[t];
        const int i = A.ti[kr], j = A.tj[kr];
        if ((A.ev[j] - A.ev[i]) * ekt > A.cut_x) {
          const double cut_rate = kr < A.nline ? A.Aji[kr] : A.bf_cut_rate;
          W[i + n * j] = W[i + n * j] + cut_rate;
          W[j + n * i] = W[j + n * i] + cut_rate * ns[j] / ns[i];
          continue;
        }
        const double th = (double)C.gij[(size_t)c + (size_t)ncell * kr];
        const double dv = (double)C.gji[(size_t)c + (size_t)ncell * kr];
        double r_up, r_down;
        if (kr < A.nline) {
          const double g_ij = A.g[i] / A.g[j];
          if (ns[i] > 0 && ns[j] > 0) {
            const double beta_ref = ns[j] * g_ij / ns[i];
            r_up = th * (beta_ref / (1.0 - beta_ref)) + dv;
            r_down = g_ij * (th / (1.0 - beta_ref) + dv);
          } else {
            r_up = 0;
            r_down = 0;
          }
        } else {
          r_up = th;
          r_down = dv;
        }
        W[j + n * i] = W[j + n * i] + r_up;
        W[i + n * j] = W[i + n * j] + r_down;
      }
      team_sync<TEAM>();
    }
    // collisions times cswitch (:806-811).  c starts at zero and takes each
    // nonzero classic rate, the electron one first (classic_col :1846-1876), then
    // every record's rates in order (gencol :2350-2351).  Without records the
    // pairs are distinct and each lane takes whole pairs; with records each lane
    // sums whole matrix elements.
    if (P.cswitch > 0 && (A.ncol > 0 || A.nel > 0)) {
      SeColCell cw{0, 0, 0, 0, 0, 0, 0, 0};
      double temp = 0, lsaha = 0;
      if (CM != 0) {
        temp = C.temp[c];
        cw = se_col_cell(temp, C.ne[c], ekt, C.dxi ? C.dxi[c] : 0.0, C.nh1 ? C.nh1[c] : 0.0);
        if (CM == 2) lsaha = C.lsaha ? C.lsaha[c] : 0.0;
      }
      auto pair_rates = [&](int p, double &ue, double &uh) {
        if (CM == 0) {
          ue = C.cup[(size_t)c + (size_t)ncell * p];
          uh = A.chkind ? C.cup[(size_t)c + (size_t)ncell * (A.ncol + p)] : 0.0;
        } else {
          se_col_rates<CM == 2>(A, cw, p, ue, uh);
        }
      };
      if (CM != 1 && A.nel > 0) {
        const int r0 = A.chkind ? 2 * A.ncol : A.ncol;
        for (int e = lane; e < A.nel; e += TEAM) {
          double cv = 0;
          for (int k = A.el_off[e]; k < A.el_off[e + 1]; k++) {
            const int code = A.el_src[k], idx = code >> 2, type = code & 3;
            if (type < 2) {
              double ue, uh;
              pair_rates(idx, ue, uh);
              if (type == 0) {
                if (ue != 0) cv = cv + ue;
                if (uh != 0) cv = cv + uh;
              } else {
                const double nij = ns[A.ci[idx]] / ns[A.cj[idx]];
                if (ue != 0) cv = cv + ue * nij;
                if (uh != 0) cv = cv + uh * nij;
              }
            } else {
              double up, dn;
              if (CM == 0) {
                up = C.cup[(size_t)c + (size_t)ncell * (r0 + idx)];
                dn = C.cup[(size_t)c + (size_t)ncell * (r0 + A.ngrec + idx)];
              } else {
                const int kc = A.gcoll ? A.gcoll[idx] : -1;
                const double nc = kc >= 0 ? C.coll[(size_t)c + (size_t)ncell * kc] : 0.0;
                se_gencol_rates(A, idx, temp, cw.ne, cw.dxi, cw.nh1, lsaha, nc, ekt, ns[A.gll[idx]],
                                ns[A.gul[idx]], up, dn);
              }
              cv = cv + (type == 2 ? up : dn);
            }
          }
          W[A.el_w[e]] = W[A.el_w[e]] + cv * P.cswitch;
        }
      } else {
        for (int p = lane; p < A.ncol; p += TEAM) {
          double ue, uh;
          pair_rates(p, ue, uh);
          if (ue == 0 && uh == 0) continue;
          const int i = A.ci[p], j = A.cj[p];
          const double nij = ns[i] / ns[j];
          double cu = 0, cd = 0;
          if (ue != 0) {
            cu = cu + ue;
            cd = cd + ue * nij;
          }
          if (uh != 0) {
            cu = cu + uh;
            cd = cd + uh * nij;
          }
          W[j + n * i] = W[j + n * i] + cu * P.cswitch;
          W[i + n * j] = W[i + n * j] + cd * P.cswitch;
        }
      }
      team_sync<TEAM>();
    }
    // diagonal = -(column sum), each lane one column
    for (int i = lane; i < n; i += TEAM) {
      double s = 0;
      for (int k = 0; k < n; k++) s = s + W[k + n * i];
      W[i + n * i] = -s;
    }
    // the conservation row: the first level of largest b n*
    int pos = 0;
    {
      double bst = bl[0] * ns[0];
      for (int k = 1; k < n; k++) {
        const double v = bl[k] * ns[k];
        if (v > bst) { bst = v; pos = k; }
      }
    }
    team_sync<TEAM>();
    for (int idx = lane; idx < n * n; idx += TEAM) {
      const int i = idx % n, j = idx / n;
      W[idx] = (i == pos) ? bl[j] * ns[j] : (W[idx] * bl[j]) * ns[j];
    }
    if (lane == 0) e[pos] = totn;
    team_sync<TEAM>();

    if constexpr (TEAM == 32) {
      if (P.solver == 1) se_solve_lineq(W, e, q, icol, n, lane);
      else if (P.solver == 2) se_solve_partial(W, e, n, lane);
      else se_solve_no_pivot(W, e, n, lane);
    } else {
      se_solve_no_pivot<TEAM>(W, e, n, lane);  // the host sends only lineq_no_pivot to larger teams
    }

    bool finite = true;
    for (int k = lane; k < n; k += TEAM) finite = finite && (fabs(e[k]) <= DBL_MAX);
    if (!team_all<TEAM>(finite)) {
      if (lane == 0) atomicMin((unsigned long long *)nonfinite, (unsigned long long)c);
      team_sync<TEAM>();
      continue;
    }
    // limiter, under-relaxation, the update
    for (int k = lane; k < n; k += TEAM) {
      double x = e[k];
      if (x < elo || x > eup) nclamp++;
      ntot++;
      if (x < elo) x = elo * exp(fmax(x, 0.0) / elo - 1.0);
      else if (x > eup) x = eup * (2.0 - eup / x);
      if (P.sor_w != 1.0) x = pow(x, P.sor_w);
      q[k] = bl[k];          // bold
      bl[k] = bl[k] * x;
    }
    team_sync<TEAM>();
    double sum = 0;
    for (int k = 0; k < n; k++) sum = sum + bl[k] * ns[k];
    const double norm = totn / sum;
    double wv = -1.0;
    int wk = -1;
    for (int k = lane, slot = 0; k < n; k += TEAM, slot++) {
      double x = bl[k] * norm;
      if (ns[k] > 0) x = fmax(x, fmin(1.0, P.min_pop_frac * totn / ns[k]));
      const double bold = q[k];
      const double ek = bold > 0 ? x / bold - 1.0 : 0.0;
      if (fabs(ek) > fabs(lv[slot])) { lv[slot] = ek; lc[slot] = c; }
      double ew = fabs(ek);
      if (P.conv_pop_floor > 0) ew = ew * fmin(1.0, x * ns[k] / (P.conv_pop_floor * totn));
      if (ew > wv) { wv = ew; wk = k; }  // a NaN never wins, as in the sequential scan
      e[k] = ek;
      C.b[(size_t)c + (size_t)ncell * k] = x;
    }
    team_argmax<TEAM>(wv, wk);
    team_sync<TEAM>();
    if (wk >= 0 && wv > best.maxerr_abs) {
      best.maxerr_abs = wv;
      best.maxerr = copysign(wv, e[wk]);
      best.cell = c;
      best.level = wk;
    }
    team_sync<TEAM>();
  }
  // per-warp partials
  if (lane == 0) wbest[gw] = best;
  for (int k = lane, slot = 0; k < n; k += TEAM, slot++) {
    lvl_val[(size_t)gw * n + k] = lv[slot];
    lvl_cell[(size_t)gw * n + k] = lc[slot];
  }
  for (int o = 16; o > 0; o >>= 1) {
    nclamp += __shfl_xor_sync(0xffffffffu, nclamp, o);
    ntot += __shfl_xor_sync(0xffffffffu, ntot, o);
  }
  if ((threadIdx.x & 31) == 0 && ntot) {
    atomicAdd(&counts[0], nclamp);
    atomicAdd(&counts[1], ntot);
  }
}

// one block: the largest change over the warps' partials, ties to the first cell
__global__ void k_stateq_finish(int nwarp, int n, const SeWarpBest *__restrict__ wbest,
                                const double *__restrict__ lvl_val, const long long *__restrict__ lvl_cell,
                                SeWarpBest *__restrict__ out_best, double *__restrict__ out_lvl) {
  __shared__ SeWarpBest sb[256];
  SeWarpBest b;
  b.maxerr_abs = 0;
  b.maxerr = 0;
  b.cell = -1;
  b.level = -1;
  b.pad = 0;
  for (int w = threadIdx.x; w < nwarp; w += blockDim.x) {
    const SeWarpBest o = wbest[w];
    if (o.cell >= 0 && (b.cell < 0 || o.maxerr_abs > b.maxerr_abs || (o.maxerr_abs == b.maxerr_abs && o.cell < b.cell)))
      b = o;
  }
  sb[threadIdx.x] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    SeWarpBest r = sb[0];
    for (int t = 1; t < (int)blockDim.x; t++) {
      const SeWarpBest o = sb[t];
      if (o.cell >= 0 && (r.cell < 0 || o.maxerr_abs > r.maxerr_abs || (o.maxerr_abs == r.maxerr_abs && o.cell < r.cell)))
        r = o;
    }
    *out_best = r;
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double v = 0;
    long long cc = -1;
    for (int w = 0; w < nwarp; w++) {
      const long long oc = lvl_cell[(size_t)w * n + k];
      const double ov = lvl_val[(size_t)w * n + k];
      if (oc >= 0 && (cc < 0 || fabs(ov) > fabs(v) || (fabs(ov) == fabs(v) && oc < cc))) { v = ov; cc = oc; }
    }
    out_lvl[k] = v;
  }
}

// ---- Ng acceleration (ng_mod.f90:241-390) ---------------------------------------
// oldb holds n1, n2, n3 as three consecutive (cell, level) blocks of nv values.

// per-block partial sums of d01, d02, d11, d12, d22, |d0|^2
__global__ void k_ng_accumulate(long long nv, const double *__restrict__ b, const double *__restrict__ oldb,
                                double *__restrict__ part) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const double n1 = log(oldb[i]), n2 = log(oldb[i + nv]), n3 = log(oldb[i + 2 * nv]), n4 = log(b[i]);
    const double d0 = n4 - n3, d1 = d0 - (n3 - n2), d2 = d0 - (n2 - n1);
    acc[0] += d0 * d1;
    acc[1] += d0 * d2;
    acc[2] += d1 * d1;
    acc[3] += d1 * d2;
    acc[4] += d2 * d2;
    acc[5] += d0 * d0;
  }
  __shared__ double red[6][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int q = 0; q < 6; q++) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0;
    for (int t = 0; t < (int)(blockDim.x >> 5); t++) v += red[threadIdx.x][t];
    part[(size_t)blockIdx.x * 6 + threadIdx.x] = v;
  }
}

__global__ void k_ng_accumulate_finish(int nblk, const double *__restrict__ part, double *__restrict__ gram) {
  if (threadIdx.x < 6) {
    double v = 0;
    for (int t = 0; t < nblk; t++) v += part[(size_t)t * 6 + threadIdx.x];
    const int q = threadIdx.x;
    // gram: d01, d02, d11, d12, d21, d22, |d0|^2
    if (q == 0) gram[0] = v;
    if (q == 1) gram[1] = v;
    if (q == 2) gram[2] = v;
    if (q == 3) { gram[3] = v; gram[4] = v; }
    if (q == 4) gram[5] = v;
    if (q == 5) gram[6] = v;
  }
}

// pass 1: the largest |ln step| per block
__global__ void k_ng_worst(long long nv, const double *__restrict__ b, const double *__restrict__ oldb, double a,
                           double bc, double *__restrict__ part) {
  double worst = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const double n2 = log(oldb[i + nv]), n3 = log(oldb[i + 2 * nv]), n4 = log(b[i]);
    const double e = (1.0 - a - bc) * n4 + a * n3 + bc * n2;
    worst = fmax(worst, fabs(e - n4));
  }
  for (int o = 16; o > 0; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int t = 0; t < (int)(blockDim.x >> 5); t++) v = fmax(v, red[t]);
    part[blockIdx.x] = v;
  }
}

// the veto (ng_mod.f90:345), written so that a NaN step is vetoed too
__global__ void k_ng_decide(int nblk, const double *__restrict__ part, double a, double bc, double max_change,
                            int *__restrict__ applied) {
  if (threadIdx.x == 0) {
    double worst = 0;
    for (int t = 0; t < nblk; t++) worst = fmax(worst, part[t]);
    *applied = (exp(worst) - 1.0 <= max_change && fabs(a) <= DBL_MAX && fabs(bc) <= DBL_MAX) ? 1 : 0;
  }
}

struct NgBest { double v; long long pos; };  // pos = cell * nlevel + level; -1 none

// pass 2, one thread per cell: the extrapolated b, renormalised
__global__ void k_ng_apply(int ncell, int nlevel, double *__restrict__ b, const double *__restrict__ oldb,
                           const double *__restrict__ nstar, const double *__restrict__ totn, double a, double bc,
                           const int *__restrict__ applied, NgBest *__restrict__ part) {
  NgBest best{0.0, -1};
  if (*applied) {
    const long long nv = (long long)ncell * nlevel;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
      for (int k = 0; k < nlevel; k++) {
        const long long i = c + (long long)ncell * k;
        const double n2 = log(oldb[i + nv]), n3 = log(oldb[i + 2 * nv]), n4 = log(b[i]);
        const double e = (1.0 - a - bc) * n4 + a * n3 + bc * n2;
        b[i] = exp(e);
        const double enew = exp(e - n4) - 1.0;
        if (fabs(enew) > fabs(best.v)) { best.v = enew; best.pos = (long long)c * nlevel + k; }
      }
      double s = 0;
      for (int k = 0; k < nlevel; k++) s = s + b[c + (long long)ncell * k] * nstar[c + (long long)ncell * k];
      const double f = totn[c] / s;
      for (int k = 0; k < nlevel; k++) b[c + (long long)ncell * k] = b[c + (long long)ncell * k] * f;
    }
  }
  // block arg-max of |enew|, ties to the first (cell, level)
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, best.v, o);
    const long long op = __shfl_xor_sync(0xffffffffu, best.pos, o);
    if (op >= 0 && (best.pos < 0 || fabs(ov) > fabs(best.v) || (fabs(ov) == fabs(best.v) && op < best.pos))) {
      best.v = ov;
      best.pos = op;
    }
  }
  __shared__ NgBest red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    NgBest r = red[0];
    for (int t = 1; t < (int)(blockDim.x >> 5); t++) {
      const NgBest o = red[t];
      if (o.pos >= 0 && (r.pos < 0 || fabs(o.v) > fabs(r.v) || (fabs(o.v) == fabs(r.v) && o.pos < r.pos))) r = o;
    }
    part[blockIdx.x] = r;
  }
}

__global__ void k_ng_apply_finish(int nblk, const NgBest *__restrict__ part, NgBest *__restrict__ out) {
  if (threadIdx.x == 0) {
    NgBest r{0.0, -1};
    for (int t = 0; t < nblk; t++) {
      const NgBest o = part[t];
      if (o.pos >= 0 && (r.pos < 0 || fabs(o.v) > fabs(r.v) || (fabs(o.v) == fabs(r.v) && o.pos < r.pos))) r = o;
    }
    *out = r;
  }
}

}  // namespace m3d

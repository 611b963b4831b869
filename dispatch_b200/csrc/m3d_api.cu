// libm3dgpu.so: the C ABI of include/m3dgpu.h over the sm_100a kernels.
//
// Host pointers are staged through device buffers for the duration of a call;
// with M3D_DEVICE_PTRS the caller's device pointers are used directly and the
// call only enqueues work on the library stream.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <sys/stat.h>

#include <cuda_runtime.h>

#include "../../include/m3dgpu.h"
#include "m3d_pipeline.cuh"
#include "m3d_stateq.cuh"
#include "m3d_nlte.cuh"
#include "m3d_aux.cuh"
#include "m3d_columns.cuh"
#include "m3d_colfused.cuh"
#include "m3d_continuum.cuh"
#include "m3d_optab.cuh"
#include "m3d_hprof.cuh"
#include "m3d_adjoint.cuh"

using namespace m3d;

namespace {

struct Ctx {
  bool init = false;
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  float *d_tgx = nullptr, *d_th2x = nullptr;
  float2 *d_tab = nullptr;  // (TGX(i), TH2X(i)) interleaved, read by the kernels
  double2 *d_tab64 = nullptr;  // the same two tables in fp64, for the plain FP64 opacity
  float *d_dW = nullptr;       // W'(u) of the TH2X table, for the adjoint (built on first use)
  std::vector<float> h_tgx, h_th2x;
  long long launches = 0;
  int se_team = 0;             // threads per cell of the last m3d_stateq_update
  std::string err;
  // scratch buffers kept between calls, grown on demand
  std::vector<void *> scratch;
  std::vector<size_t> scratch_bytes;
  // staging buffers of host-pointer calls, reused from call to call
  std::vector<void *> stage_buf;
  std::vector<size_t> stage_bytes;
  // stage timing (m3d_profile_enable)
  bool profile = false;
  std::vector<cudaEvent_t> ev_free;
  struct Rec { int stage; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  double stage_ms[4] = {0, 0, 0, 0};
  long long stage_n[4] = {0, 0, 0, 0};
  // device allocations this context has made (m3d_alloc_stats)
  long long mallocs = 0;
};

// One context per host thread: a thread that calls m3d_init gets its own stream,
// scratch and staging buffers, QLG tables, error string and counters, so slabs
// handled by different host threads run concurrently on their own streams.
thread_local Ctx g_ctx;

// every device allocation of the library goes through here and is counted
template <typename T>
cudaError_t dev_malloc(T **p, size_t bytes) {
  g_ctx.mallocs++;
  return cudaMalloc(reinterpret_cast<void **>(p), bytes);
}

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_ctx.err = buf;
  return code;
}

#define CUDA_TRY(expr)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) return fail(M3D_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

cudaEvent_t take_event() {
  if (!g_ctx.ev_free.empty()) {
    cudaEvent_t e = g_ctx.ev_free.back();
    g_ctx.ev_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

#define LAUNCH_S(stage_, kernel, grid, block, smem, ...)                                           \
  do {                                                                                             \
    cudaEvent_t ea_ = nullptr, eb_ = nullptr;                                                      \
    if (g_ctx.profile) {                                                                           \
      ea_ = take_event();                                                                          \
      eb_ = take_event();                                                                          \
      cudaEventRecord(ea_, g_ctx.stream);                                                          \
    }                                                                                              \
    kernel<<<(grid), (block), (smem), g_ctx.stream>>>(__VA_ARGS__);                                \
    g_ctx.launches++;                                                                              \
    cudaError_t e_ = cudaGetLastError();                                                           \
    if (e_ != cudaSuccess) return fail(M3D_ECUDA, "launch %s: %s", #kernel, cudaGetErrorString(e_)); \
    if (g_ctx.profile) {                                                                           \
      cudaEventRecord(eb_, g_ctx.stream);                                                          \
      g_ctx.recs.push_back(Ctx::Rec{(stage_), ea_, eb_});                                          \
    }                                                                                              \
  } while (0)
#define LAUNCH(kernel, grid, block, smem, ...) LAUNCH_S(M3D_STAGE_OTHER, kernel, grid, block, smem, __VA_ARGS__)

int need_init() {
  if (!g_ctx.init) return fail(M3D_ENOINIT, "m3d_init has not been called");
  return M3D_OK;
}

// scratch slot: a device buffer of at least `bytes`, kept for later calls
int scratch(int slot, size_t bytes, void **out) {
  if ((int)g_ctx.scratch.size() <= slot) {
    g_ctx.scratch.resize(slot + 1, nullptr);
    g_ctx.scratch_bytes.resize(slot + 1, 0);
  }
  if (g_ctx.scratch_bytes[slot] < bytes) {
    if (g_ctx.scratch[slot]) {
      CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
      CUDA_TRY(cudaFree(g_ctx.scratch[slot]));
      g_ctx.scratch[slot] = nullptr;
      g_ctx.scratch_bytes[slot] = 0;
    }
    CUDA_TRY(dev_malloc(&g_ctx.scratch[slot], bytes));
    g_ctx.scratch_bytes[slot] = bytes;
  }
  *out = g_ctx.scratch[slot];
  return M3D_OK;
}

// Host-pointer staging for one call: device copies of the arguments, copied
// back on finish() for the ones marked out.
class Staging {
 public:
  explicit Staging(unsigned flags) : dev_(flags & M3D_DEVICE_PTRS) {}
  // in: copied to the device; out: copied back; both: both
  template <typename T>
  int map(T *host, size_t count, bool in, bool out, T **dptr) {
    if (host == nullptr || count == 0) { *dptr = nullptr; return M3D_OK; }
    if (dev_) { *dptr = host; return M3D_OK; }
    Buf b;
    b.host = (void *)host;
    b.bytes = count * sizeof(T);
    b.out = out;
    const size_t slot = bufs_.size();
    if (g_ctx.stage_buf.size() <= slot) {
      g_ctx.stage_buf.resize(slot + 1, nullptr);
      g_ctx.stage_bytes.resize(slot + 1, 0);
    }
    if (g_ctx.stage_bytes[slot] < b.bytes) {
      if (g_ctx.stage_buf[slot]) {
        CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
        CUDA_TRY(cudaFree(g_ctx.stage_buf[slot]));
      }
      g_ctx.stage_buf[slot] = nullptr;
      g_ctx.stage_bytes[slot] = 0;
      CUDA_TRY(dev_malloc(&g_ctx.stage_buf[slot], b.bytes));
      g_ctx.stage_bytes[slot] = b.bytes;
    }
    b.dptr = g_ctx.stage_buf[slot];
    if (in) CUDA_TRY(cudaMemcpyAsync(b.dptr, host, b.bytes, cudaMemcpyHostToDevice, g_ctx.stream));
    else CUDA_TRY(cudaMemsetAsync(b.dptr, 0, b.bytes, g_ctx.stream));
    bufs_.push_back(b);
    *dptr = (T *)b.dptr;
    return M3D_OK;
  }
  template <typename T>
  int in(const T *host, size_t count, const T **dptr) {
    T *d;
    int rc = map(const_cast<T *>(host), count, true, false, &d);
    *dptr = d;
    return rc;
  }
  int finish() {
    if (dev_) return M3D_OK;
    for (auto &b : bufs_)
      if (b.out) CUDA_TRY(cudaMemcpyAsync(b.host, b.dptr, b.bytes, cudaMemcpyDeviceToHost, g_ctx.stream));
    CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
    return M3D_OK;
  }
  bool device() const { return dev_; }

 private:
  struct Buf { void *dptr = nullptr; void *host = nullptr; size_t bytes = 0; bool out = false; };
  bool dev_;
  std::vector<Buf> bufs_;
};

#define TRY(expr)                  \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != M3D_OK) return rc_; \
  } while (0)

int wrap_host(int v, int n) { v %= n; return v < 0 ? v + n : v; }
int grid_for(size_t n, int block = 256) {
  size_t g = (n + block - 1) / block;
  const size_t cap = (size_t)148 * 32;
  return (int)(g > cap ? cap : (g < 1 ? 1 : g));
}

// ---- QLG tables: qlg_init (qlg_mod.f90:364-375) with the Weideman-32 /
// Humlicek-w4 fp64 reference (qlg_mod.f90:411-447) and Z_0.2 (qlg_mod.f90:384-399)
const double W32_LD = 4.75682846001088411e+00;
const double W32_AD[32] = {
    -1.30317978630500875e-12, +3.74107755472269789e-12, +8.03033538228436012e-12, -2.15435373143760700e-11,
    -5.54423561143486540e-11, +1.16582546820233235e-10, +4.15374271614691897e-10, -5.23102143724924582e-10,
    -3.20801514078875819e-09, +8.12488896568210460e-10, +2.37975567593842971e-08, +2.29304391194392872e-08,
    -1.48130789124396946e-07, -4.18407637053084035e-07, +4.25583313792292626e-07, +4.40153173159092505e-06,
    +6.82103194402497841e-06, -2.14096192018698432e-05, -1.30754492546239731e-04, -2.45329802700202065e-04,
    +3.92591360700705167e-04, +4.51954110534923473e-03, +1.90061557848454077e-02, +5.73044035298371918e-02,
    +1.40607162268937713e-01, +2.95444510715087261e-01, +5.46013972063934205e-01, +9.01925489364799993e-01,
    +1.34554416923454490e+00, +1.82566962963248147e+00, +2.26353729990026764e+00, +2.57225340812456960e+00};

double voigt_ref_f64(double a, double v) {
  const double ISQPI8 = 0.564189583547756287;
  const double av = fabs(v);
  if (av + a >= 15.0) {
    const double tr = a * a - av * av + 0.5, ti = -2.0 * a * av;
    const double q = 1.0 / (tr * tr + ti * ti);
    return ISQPI8 * ((a * tr + (-av) * ti) * q);
  }
  const double dr = W32_LD + a, nr0 = W32_LD - a, di = -v;
  const double q = 1.0 / (dr * dr + di * di);
  const double zr = (nr0 * dr + v * di) * q, zi = (v * dr - nr0 * di) * q;
  double pr = W32_AD[0], pim = 0.0;
  for (int j = 1; j < 32; j++) {
    const double t = pr * zr - pim * zi + W32_AD[j];
    pim = pr * zi + pim * zr;
    pr = t;
  }
  const double ir = dr * q, ii = -di * q;
  const double sr = ir * ir - ii * ii, si = 2.0 * ir * ii;
  return 2.0 * (pr * sr - pim * si) + ISQPI8 * ir;
}

double z02_over_l2(double u) {
  const double A2 = 0.18741813853432507, GAM = 0.93709069267162530, KP = 0.81924853602069690;
  const double ETA = 0.14697983683153040, QRS = 0.16, DLN2 = 0.69314718055994531;
  const double v = GAM * sqrt(u), L = 1.0 / (1.0 + u), G = exp(-DLN2 * u);
  const double Kv = voigt_ref_f64(A2, v);
  const double P = KP * (ETA * L + (1.0 - ETA) * G);
  return (Kv - P) / (QRS * KP) * (1.0 + u) * (1.0 + u);
}

int ensure_tables() {
  if (g_ctx.d_tgx) return M3D_OK;
  g_ctx.h_tgx.resize(QLG_NTAB);
  g_ctx.h_th2x.resize(QLG_NTAB);
  for (int i = 0; i < QLG_NTAB; i++) {
    const double x = (double)i / 800.0;
    g_ctx.h_tgx[i] = (float)pow(2.0, -x * x);
    g_ctx.h_th2x[i] = (float)z02_over_l2(x * x);
  }
  CUDA_TRY(dev_malloc(&g_ctx.d_tgx, 2 * QLG_NTAB * sizeof(float)));
  g_ctx.d_th2x = g_ctx.d_tgx + QLG_NTAB;
  CUDA_TRY(cudaMemcpy(g_ctx.d_tgx, g_ctx.h_tgx.data(), QLG_NTAB * sizeof(float), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(g_ctx.d_th2x, g_ctx.h_th2x.data(), QLG_NTAB * sizeof(float), cudaMemcpyHostToDevice));
  std::vector<float2> tab(QLG_NTAB);
  for (int i = 0; i < QLG_NTAB; i++) tab[i] = make_float2(g_ctx.h_tgx[i], g_ctx.h_th2x[i]);
  CUDA_TRY(dev_malloc(&g_ctx.d_tab, QLG_NTAB * sizeof(float2)));
  CUDA_TRY(cudaMemcpy(g_ctx.d_tab, tab.data(), QLG_NTAB * sizeof(float2), cudaMemcpyHostToDevice));
  std::vector<double2> tab64(QLG_NTAB);
  for (int i = 0; i < QLG_NTAB; i++) {
    const double x = (double)i / 800.0;
    tab64[i] = make_double2(pow(2.0, -x * x), z02_over_l2(x * x));
  }
  CUDA_TRY(dev_malloc(&g_ctx.d_tab64, QLG_NTAB * sizeof(double2)));
  CUDA_TRY(cudaMemcpy(g_ctx.d_tab64, tab64.data(), QLG_NTAB * sizeof(double2), cudaMemcpyHostToDevice));
  return M3D_OK;
}

SlabArgs slab_args(const m3d_slab_t *s, unsigned flags) {
  SlabArgs a;
  a.nf = s->nf; a.nx = s->nx; a.ny = s->ny; a.nz = s->nz; a.dir = s->dir;
  a.get_psi = s->get_psi || (flags & M3D_GET_PSI);
  a.split_rates = s->split_rates || (flags & M3D_SPLIT_RATES);
  for (int i = 0; i < 3; i++) { a.ds[i] = s->ds[i]; a.vec[i] = s->vec[i]; }
  a.maser_dtau_max = s->maser_dtau_max;
  a.maser_Inu_max = s->maser_Inu_max;
  return a;
}

int check_slab(const m3d_slab_t *s) {
  if (!s) return fail(M3D_EINVAL, "slab is NULL");
  if (s->nf < 1 || s->nx < 1 || s->ny < 1 || s->nz < 2) return fail(M3D_EINVAL, "slab needs nf,nx,ny >= 1 and nz >= 2");
  if (s->dir != 1 && s->dir != -1) return fail(M3D_EINVAL, "slab dir must be +1 or -1");
  if (s->vec[2] == 0.0) return fail(M3D_EINVAL, "ray direction with vec(3) = 0");
  return M3D_OK;
}

// set_stencil (ray_mod.f90:493-512) and the Keys kernel (ray_mod.f90:581-597)
void cc_kernel(double s, double k[4]) {
  const double s2 = s * s, s3 = s2 * s;
  k[0] = 0.5 * (-s3 + 2 * s2 - s);
  k[1] = 0.5 * (3 * s3 - 5 * s2 + 2);
  k[2] = 0.5 * (-3 * s3 + 4 * s2 + s);
  k[3] = 0.5 * (s3 - s2);
}
void set_stencil(const double ds[3], const double vec[3], double xk[4], double yk[4], int *upo1, int *upo2,
                 double *dsup) {
  *dsup = ds[2] / fabs(vec[2]);
  const double wt1 = -vec[0] / ds[0] * *dsup, wt2 = -vec[1] / ds[1] * *dsup;
  const double h1 = wt1 > 0 ? wt1 : wt1 + 1, h2 = wt2 > 0 ? wt2 : wt2 + 1;
  *upo1 = wt1 > 0 ? -1 : -2;
  *upo2 = wt2 > 0 ? -1 : -2;
  cc_kernel(h1, xk);
  cc_kernel(h2, yk);
}

// quadratic solver constants (rt_solvers_mod.f90:908-912)
QuadConst quad_const(double ds_cm3, double vec3) {
  QuadConst q;
  const float ds = (float)ds_cm3;
  const float dsup = (float)((double)ds / fabs(vec3));
  q.rdsup = 1.0f / dsup;
  q.dsup1 = 0.5f * dsup;
  q.dsup2 = ((1.0f / 12.0f) * dsup) * dsup;
  return q;
}

// pchip_mono extrapolation constants for the bottom ghost (interpol_mod.f90:289-365
// with xx = (1,2,3)*ds, newx = 0)
PchipConst pchip_const(float ds3_code) {
  PchipConst c;
  const float xx1 = (float)(1.0 * (double)ds3_code), xx2 = (float)(2.0 * (double)ds3_code);
  c.dx1 = xx2 - xx1;
  const float t1 = (0.0f - xx1) / c.dx1;
  const float t2 = t1 * t1, t3 = t2 * t1;
  c.p = 3.0f * t2 - 2.0f * t3;
  c.c0 = 1.0f - c.p;
  c.cm0 = (t3 - 2.0f * t2) + t1;
  c.cm1 = t3 - t2;
  return c;
}

// rotate_array coefficients of local plane z of a slab (rt_patch_mod.f90:3821-3841).
// rot_planes and the no-allocation rotation both take their weights from here.
RotPlane rot_plane_at(const double vec[3], const double ds_code[3], double bot2pivot, const double ray_offset[2],
                      int z) {
  const float delta0 = (float)(vec[0] / (vec[2] * ds_code[0]));
  const float delta1 = (float)(vec[1] / (vec[2] * ds_code[1]));
  const float b2p = (float)bot2pivot;
  const float height = (float)((double)z * ds_code[2]);
  const float dk0 = (float)((double)((b2p - height) * delta0) + ray_offset[0]);
  const float dk1 = (float)((double)((b2p - height) * delta1) + ray_offset[1]);
  const int up1 = (int)floorf(dk0), up2 = (int)floorf(dk1);
  const float f1 = dk0 - (float)up1, f2 = dk1 - (float)up2;
  RotPlane r;
  r.up1 = up1;
  r.up2 = up2;
  r.a = (1.0f - f1) * (1.0f - f2);
  r.b = f1 * (1.0f - f2);
  r.c = (1.0f - f1) * f2;
  r.d = f1 * f2;
  return r;
}

// the weights of local planes 1..nz
void rot_planes(const double vec[3], const double ds_code[3], double bot2pivot, const double ray_offset[2], int nz,
                RotPlane *out) {
  for (int z = 1; z <= nz; z++) out[z - 1] = rot_plane_at(vec, ds_code, bot2pivot, ray_offset, z);
}

LineArgs line_args(const m3d_linelist_t *ll) {
  LineArgs L;
  L.nline = ll->nline;
  L.llam0 = ll->llam0;
  L.lower_ev = ll->lower_ev; L.gpref = ll->gpref; L.grad = ll->grad;
  L.gw1 = ll->gw1; L.gw2 = ll->gw2; L.gstk = ll->gstk;
  L.unsold = ll->unsold;
  L.lev_i = ll->lev_i; L.lev_j = ll->lev_j;
  L.active = ll->active;
  L.reach_in = ll->reach_in;
  L.sel = nullptr;
  L.nsel = nullptr;
  return L;
}

// stage a line list's arrays
int stage_linelist(Staging &st, const m3d_linelist_t *ll, LineArgs *L) {
  const size_t n = (size_t)ll->nline;
  *L = line_args(ll);
  TRY(st.in(ll->llam0, n, &L->llam0));
  TRY(st.in(ll->lower_ev, n, &L->lower_ev));
  TRY(st.in(ll->gpref, n, &L->gpref));
  TRY(st.in(ll->grad, n, &L->grad));
  TRY(st.in(ll->gw1, n, &L->gw1));
  TRY(st.in(ll->gw2, n, &L->gw2));
  TRY(st.in(ll->gstk, n, &L->gstk));
  TRY(st.in(ll->unsold, n, &L->unsold));
  TRY(st.in(ll->lev_i, n, &L->lev_i));
  TRY(st.in(ll->lev_j, n, &L->lev_j));
  TRY(st.in(ll->active, n, &L->active));
  TRY(st.in(ll->reach_in, n, &L->reach_in));
  if (!L->llam0 || !L->lower_ev || !L->gpref || !L->grad || !L->gw1 || !L->gw2 || !L->gstk || !L->unsold)
    return fail(M3D_EINVAL, "line list with a NULL array");
  return M3D_OK;
}

GridArgs grid_args(int nf, const double *llam_host_or_dev, const double *d_llam, bool dev, float tol,
                   float line_reject_frac) {
  GridArgs G;
  double l0, l1;
  if (dev) {
    cudaMemcpy(&l0, llam_host_or_dev, sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(&l1, llam_host_or_dev + nf - 1, sizeof(double), cudaMemcpyDeviceToHost);
  } else {
    l0 = llam_host_or_dev[0];
    l1 = llam_host_or_dev[nf - 1];
  }
  G.nf = nf;
  G.llam = d_llam;
  G.llam1 = l0;
  G.dllam = (l1 - l0) / (double)(nf - 1);
  G.inv_dllam = 1.0 / G.dllam;
  G.sdl = (float)G.inv_dllam;
  G.tol = tol;
  G.flo_scale = fmaxf(tol, line_reject_frac) * tol;
  return G;
}

}  // namespace

// ============================================================================
extern "C" {

int m3d_init(int device, unsigned flags) {
  (void)flags;
  if (g_ctx.init) {
    if (device != g_ctx.device) return fail(M3D_EINVAL, "already initialised on device %d", g_ctx.device);
    return M3D_OK;
  }
  int n = 0;
  CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(M3D_EINVAL, "device %d not present (%d devices)", device, n);
  CUDA_TRY(cudaSetDevice(device));
  CUDA_TRY(cudaStreamCreateWithFlags(&g_ctx.own, cudaStreamNonBlocking));
  g_ctx.stream = g_ctx.own;
  g_ctx.device = device;
  g_ctx.init = true;
  return ensure_tables();
}

int m3d_free(void) {
  if (!g_ctx.init) return M3D_OK;
  cudaStreamSynchronize(g_ctx.stream);
  for (void *p : g_ctx.scratch) if (p) cudaFree(p);
  g_ctx.scratch.clear();
  g_ctx.scratch_bytes.clear();
  for (void *p : g_ctx.stage_buf) if (p) cudaFree(p);
  g_ctx.stage_buf.clear();
  g_ctx.stage_bytes.clear();
  for (auto &r : g_ctx.recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  g_ctx.recs.clear();
  for (auto e : g_ctx.ev_free) cudaEventDestroy(e);
  g_ctx.ev_free.clear();
  if (g_ctx.d_tgx) cudaFree(g_ctx.d_tgx);
  g_ctx.d_tgx = g_ctx.d_th2x = nullptr;
  if (g_ctx.d_tab) cudaFree(g_ctx.d_tab);
  g_ctx.d_tab = nullptr;
  if (g_ctx.d_tab64) cudaFree(g_ctx.d_tab64);
  g_ctx.d_tab64 = nullptr;
  if (g_ctx.d_dW) cudaFree(g_ctx.d_dW);
  g_ctx.d_dW = nullptr;
  if (g_ctx.own) cudaStreamDestroy(g_ctx.own);
  g_ctx.own = g_ctx.stream = nullptr;
  g_ctx.init = false;
  g_ctx.mallocs = 0;
  return M3D_OK;
}

int m3d_last_error(char *buf, int buflen) {
  if (!buf || buflen < 1) return M3D_EINVAL;
  snprintf(buf, (size_t)buflen, "%s", g_ctx.err.c_str());
  return M3D_OK;
}

int m3d_version(int *major, int *minor, int *patch) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  if (patch) *patch = 0;
  return M3D_OK;
}

int m3d_set_stream(void *s) {
  TRY(need_init());
  g_ctx.stream = s ? (cudaStream_t)s : g_ctx.own;
  return M3D_OK;
}

int m3d_synchronize(void) {
  TRY(need_init());
  CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  return M3D_OK;
}

long long m3d_launch_count(void) { return g_ctx.launches; }

int m3d_alloc_stats(long long *mallocs, unsigned long long *scratch_bytes, unsigned long long *staging_bytes) {
  unsigned long long sb = 0, tb = 0;
  for (size_t b : g_ctx.scratch_bytes) sb += b;
  for (size_t b : g_ctx.stage_bytes) tb += b;
  if (mallocs) *mallocs = g_ctx.mallocs;
  if (scratch_bytes) *scratch_bytes = sb;
  if (staging_bytes) *staging_bytes = tb;
  return M3D_OK;
}

int m3d_profile_enable(int on) {
  TRY(need_init());
  g_ctx.profile = on != 0;
  for (int i = 0; i < 4; i++) { g_ctx.stage_ms[i] = 0; g_ctx.stage_n[i] = 0; }
  return M3D_OK;
}

int m3d_profile_read(int stage, double *ms, long long *launches) {
  TRY(need_init());
  if (stage < 0 || stage > 3) return fail(M3D_EINVAL, "m3d_profile_read: stage %d", stage);
  CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  for (auto &r : g_ctx.recs) {
    float t = 0;
    CUDA_TRY(cudaEventElapsedTime(&t, r.a, r.b));
    g_ctx.stage_ms[r.stage] += t;
    g_ctx.stage_n[r.stage] += 1;
    g_ctx.ev_free.push_back(r.a);
    g_ctx.ev_free.push_back(r.b);
  }
  g_ctx.recs.clear();
  if (ms) *ms = g_ctx.stage_ms[stage];
  if (launches) *launches = g_ctx.stage_n[stage];
  return M3D_OK;
}

int m3d_weights(int which, int n, const void *t, void *o1, void *o2, void *o3, void *o4, unsigned flags) {
  TRY(need_init());
  if (n < 0 || which < 0 || which > 5) return fail(M3D_EINVAL, "m3d_weights: bad which/n");
  if (n == 0) return M3D_OK;
  const bool f64 = flags & M3D_FP64;
  if (f64 && which != 1 && which != 2) return fail(M3D_EUNSUPPORTED, "m3d_weights: FP64 has which = 1, 2 only");
  const int nout = which == 0 ? 2 : ((which == 3 || which == 4) ? 1 : 4);
  Staging st(flags);
  if (f64) {
    const double *dt; double *d[4] = {nullptr, nullptr, nullptr, nullptr};
    TRY(st.in((const double *)t, n, &dt));
    void *outs[4] = {o1, o2, o3, o4};
    for (int i = 0; i < nout; i++) TRY(st.map((double *)outs[i], n, false, true, &d[i]));
    LAUNCH(k_weights_f64, grid_for(n), 256, 0, which, n, dt, d[0], d[1], d[2], d[3]);
  } else {
    const float *dt; float *d[4] = {nullptr, nullptr, nullptr, nullptr};
    TRY(st.in((const float *)t, n, &dt));
    void *outs[4] = {o1, o2, o3, o4};
    for (int i = 0; i < nout; i++) TRY(st.map((float *)outs[i], n, false, true, &d[i]));
    LAUNCH(k_weights_f32, grid_for(n), 256, 0, which, n, dt, d[0], d[1], d[2], d[3]);
  }
  return st.finish();
}

int m3d_qlg_init(void) {
  TRY(need_init());
  return ensure_tables();
}

int m3d_qlg_tables(float *tgx, float *th2x) {
  TRY(need_init());
  TRY(ensure_tables());
  if (tgx) memcpy(tgx, g_ctx.h_tgx.data(), QLG_NTAB * sizeof(float));
  if (th2x) memcpy(th2x, g_ctx.h_th2x.data(), QLG_NTAB * sizeof(float));
  return M3D_OK;
}

int m3d_qlg_bot_profile(int n, const float *a, const float *q, const float *vpr, const float *idf, float *h,
                        unsigned flags) {
  TRY(need_init());
  if (n < 0) return fail(M3D_EINVAL, "n < 0");
  if (n == 0) return M3D_OK;
  Staging st(flags);
  const float *da, *dq, *dv, *di;
  float *dh;
  TRY(st.in(a, n, &da)); TRY(st.in(q, n, &dq)); TRY(st.in(vpr, n, &dv)); TRY(st.in(idf, n, &di));
  TRY(st.map(h, n, false, true, &dh));
  LAUNCH(k_qlg_profile, grid_for(n), 256, 0, n, g_ctx.d_tab, da, dq, dv, di, dh);
  return st.finish();
}

int m3d_line_opacity(const m3d_linelist_t *ll, int nf, const double *llam, int ncell, float *chi, float *eta,
                     const float *cont, const float *logref, const float *vproj, const float *inv_df,
                     const float *vbar2, const float *e_kT, const float *lnbase, const float *ne,
                     const float *tothi, const float *stark_pe, const float *dep_mem, int nlevel, int do_nlte,
                     float tol, float line_reject_frac, unsigned char *used, float *strength, float *reach,
                     unsigned flags) {
  return m3d_line_opacity_scat(ll, nf, llam, ncell, chi, eta, cont, logref, vproj, inv_df, vbar2, e_kT, lnbase, ne,
                               tothi, stark_pe, dep_mem, nlevel, do_nlte, tol, line_reject_frac, used, strength,
                               reach, nullptr, nullptr, flags);
}

int m3d_line_opacity_scat(const m3d_linelist_t *ll, int nf, const double *llam, int ncell, float *chi, float *eta,
                          const float *cont, const float *logref, const float *vproj, const float *inv_df,
                          const float *vbar2, const float *e_kT, const float *lnbase, const float *ne,
                          const float *tothi, const float *stark_pe, const float *dep_mem, int nlevel, int do_nlte,
                          float tol, float line_reject_frac, unsigned char *used, float *strength, float *reach,
                          const float *one_m_eps, float *chi_scat, unsigned flags) {
  TRY(need_init());
  if ((one_m_eps == nullptr) != (chi_scat == nullptr))
    return fail(M3D_EINVAL, "m3d_line_opacity_scat: give both one_m_eps and chi_scat, or neither");
  if (!ll || !llam) return fail(M3D_EINVAL, "m3d_line_opacity: NULL line list or grid");
  if (ll->nline == 0 || nf < 2 || ncell == 0) return M3D_OK;
  if (ncell < 0 || ll->nline < 0) return fail(M3D_EINVAL, "m3d_line_opacity: negative size");
  const bool diag = flags & M3D_LINE_DIAG;
  if (diag && (!used || !strength || !reach)) return fail(M3D_EINVAL, "M3D_LINE_DIAG needs used, strength, reach");
  if (do_nlte && (!dep_mem || nlevel < 1)) return fail(M3D_EINVAL, "do_nlte needs dep_mem and nlevel");
  Staging st(flags);
  LineArgs L;
  TRY(stage_linelist(st, ll, &L));
  const double *dllam;
  TRY(st.in(llam, nf, &dllam));
  const size_t nfc = (size_t)nf * ncell;
  float *dchi, *deta;
  const float *dcont, *dlr, *dvp, *didf, *dvb, *dek, *dlb, *dne, *dth, *dsp, *ddep = nullptr;
  TRY(st.map(chi, nfc, true, true, &dchi));
  TRY(st.map(eta, nfc, true, true, &deta));
  TRY(st.in(cont, nfc, &dcont)); TRY(st.in(logref, nfc, &dlr));
  TRY(st.in(vproj, ncell, &dvp)); TRY(st.in(inv_df, ncell, &didf)); TRY(st.in(vbar2, ncell, &dvb));
  TRY(st.in(e_kT, ncell, &dek)); TRY(st.in(lnbase, ncell, &dlb)); TRY(st.in(ne, ncell, &dne));
  TRY(st.in(tothi, ncell, &dth)); TRY(st.in(stark_pe, ncell, &dsp));
  if (do_nlte) TRY(st.in(dep_mem, (size_t)ncell * nlevel, &ddep));
  const float *dome = nullptr;
  float *dcs = nullptr;
  if (chi_scat) {
    TRY(st.in(one_m_eps, nfc, &dome));
    TRY(st.map(chi_scat, nfc, true, true, &dcs));
  }
  unsigned char *dused = nullptr;
  float *dstr = nullptr, *dreach = nullptr;
  if (diag) {
    TRY(st.map(used, ll->nline, true, true, &dused));
    TRY(st.map(strength, ll->nline, true, true, &dstr));
    TRY(st.map(reach, ll->nline, true, true, &dreach));
  }
  GridArgs G = grid_args(nf, llam, dllam, st.device(), tol, line_reject_frac);
  if (!(G.dllam > 0)) return fail(M3D_EINVAL, "m3d_line_opacity: log(lambda) grid must be ascending");
  const int block = 256, warps = block / 32;
  const size_t smem = 2 * QLG_NTAB * sizeof(float);
  thread_local bool attr = false;
  if (!attr) {
    CUDA_TRY(cudaFuncSetAttribute(k_line_opacity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  if (L.reach_in) {
    // select_lines: max |vproj| over the cells, then the kept lines
    void *sp = nullptr;
    TRY(scratch(20, sizeof(int) * ((size_t)ll->nline + 8), &sp));
    unsigned *vmax = (unsigned *)sp;
    int *dnsel = (int *)sp + 1, *dsel = (int *)sp + 4;
    CUDA_TRY(cudaMemsetAsync(vmax, 0, sizeof(unsigned), g_ctx.stream));
    LAUNCH(k_absmax, grid_for(ncell), 256, 0, ncell, dvp, vmax);
    LAUNCH(k_select_lines, 1, 32, 0, L, dllam, nf, (const unsigned *)vmax, dsel, dnsel);
    L.sel = dsel;
    L.nsel = dnsel;
  }
  int grid = (ncell + warps - 1) / warps;
  if (grid > 148 * 8) grid = 148 * 8;
  LAUNCH_S(M3D_STAGE_OPACITY, k_line_opacity, grid, block, smem, L, G, ncell, dchi, deta, dcont, dlr, dvp, didf, dvb, dek, dlb, dne, dth,
         dsp, ddep, do_nlte, diag ? 1 : 0, dused, dstr, dreach, g_ctx.d_tab, dome, dcs);
  return st.finish();
}

int m3d_lte_background(int nf, int ncell, const double *nu, const float *temp, float *beta, float *Bnu,
                       unsigned flags) {
  TRY(need_init());
  if (nf < 1 || ncell < 1) return fail(M3D_EINVAL, "m3d_lte_background: empty");
  Staging st(flags);
  const double *dnu;
  const float *dt;
  float *db, *dB;
  const size_t n = (size_t)nf * ncell;
  TRY(st.in(nu, nf, &dnu)); TRY(st.in(temp, ncell, &dt));
  TRY(st.map(beta, n, false, true, &db)); TRY(st.map(Bnu, n, false, true, &dB));
  LAUNCH(k_lte_background, grid_for(n), 256, 0, nf, ncell, dnu, dt, db, dB);
  return st.finish();
}

int m3d_work_to_transfer_units(int nf, int ncell, float *w1, float *w2, const float *beta, double maser_chi_floor,
                               int suppress_masers, int *n_floored, unsigned flags) {
  TRY(need_init());
  if (nf < 1 || ncell < 1) return fail(M3D_EINVAL, "m3d_work_to_transfer_units: empty");
  Staging st(flags);
  const size_t n = (size_t)nf * ncell;
  float *d1, *d2;
  const float *db;
  int *dcnt;
  TRY(st.map(w1, n, true, true, &d1)); TRY(st.map(w2, n, true, true, &d2)); TRY(st.in(beta, n, &db));
  void *cnt;
  TRY(scratch(0, sizeof(int), &cnt));
  dcnt = (int *)cnt;
  CUDA_TRY(cudaMemsetAsync(dcnt, 0, sizeof(int), g_ctx.stream));
  LAUNCH(k_transfer_units, grid_for(n), 256, 0, n, d1, d2, db, (float)maser_chi_floor, suppress_masers, dcnt);
  if (n_floored) {
    if (st.device()) {
      CUDA_TRY(cudaMemcpyAsync(n_floored, dcnt, sizeof(int), cudaMemcpyDeviceToDevice, g_ctx.stream));
    } else {
      CUDA_TRY(cudaMemcpyAsync(n_floored, dcnt, sizeof(int), cudaMemcpyDeviceToHost, g_ctx.stream));
    }
  }
  return st.finish();
}

int m3d_integrate_intensity(int n, float wmu, const float *inu, const float *psi, float *Jnu, float *PsiJ,
                            unsigned flags) {
  TRY(need_init());
  if (n < 1) return M3D_OK;
  Staging st(flags);
  const float *di, *dp = nullptr;
  float *dJ, *dPJ = nullptr;
  TRY(st.in(inu, n, &di));
  TRY(st.map(Jnu, n, true, true, &dJ));
  if (psi && PsiJ) {
    TRY(st.in(psi, n, &dp));
    TRY(st.map(PsiJ, n, true, true, &dPJ));
  }
  LAUNCH(k_integrate_intensity, grid_for(n), 256, 0, (size_t)n, wmu, di, dp, dJ, dPJ);
  return st.finish();
}

}  // extern "C"

namespace {

template <typename T>
int rotate_impl(const m3d_slab_t *s, T *dwork, const double *ds_code, double bot2pivot, const double *ray_offset) {
  const int nf = s->nf, nx = s->nx, ny = s->ny, nz = s->nz;
  std::vector<RotPlane> h(nz);
  const double off0[2] = {0.0, 0.0};
  rot_planes(s->vec, ds_code, bot2pivot, ray_offset ? ray_offset : off0, nz, h.data());
  void *drot, *tmp;
  TRY(scratch(1, sizeof(RotPlane) * nz, &drot));
  const size_t plane = (size_t)nf * nx * ny;
  TRY(scratch(2, sizeof(T) * plane * nz * 2, &tmp));
  CUDA_TRY(cudaMemcpyAsync(drot, h.data(), sizeof(RotPlane) * nz, cudaMemcpyHostToDevice, g_ctx.stream));
  // rotate slot 0 planes 1..nz and slot 1 planes 1..nz: both views are contiguous
  for (int k = 0; k < 2; k++) {
    T *src = dwork + plane * (1 + (size_t)k * (nz + 2));
    LAUNCH_S(M3D_STAGE_SOLVE, k_rotate_planes<T>, grid_for(plane * nz), 256, 0, nf, nx, ny, nz, (const T *)src,
           (T *)tmp + plane * nz * k, (const RotPlane *)drot);
  }
  for (int k = 0; k < 2; k++)
    CUDA_TRY(cudaMemcpyAsync(dwork + plane * (1 + (size_t)k * (nz + 2)), (T *)tmp + plane * nz * k,
                             sizeof(T) * plane * nz, cudaMemcpyDeviceToDevice, g_ctx.stream));
  CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  return M3D_OK;
}

template <typename T>
int solve_impl(int solver, const m3d_slab_t *s, unsigned flags, T *work, T *psi, T *irem, T *esc,
               const float *chi500, const float *chi500_up, const float *g500, const int *eta_row,
               const unsigned char *eta_mask) {
  const SlabArgs a = slab_args(s, flags);
  const size_t ncol = (size_t)a.nf * a.nx * a.ny;
  if (a.get_psi && !psi) return fail(M3D_EINVAL, "get_psi without psi");
  if (a.split_rates && (!irem || !esc)) return fail(M3D_EINVAL, "split_rates without irem/escape");
  const int block = 256;
  const int grid = (int)((ncol + block - 1) / block);
  switch (solver) {
    case M3D_SOLVER_LINEAR: {
      const float ds = (float)s->ds[2];
      const T dsup05 = (T)((double)(0.5f * ds) / fabs(s->vec[2]));
      LAUNCH_S(M3D_STAGE_SOLVE, k_long_char_linear<T>, grid, block, 0, a, work, psi, irem, esc, dsup05);
      return M3D_OK;
    }
    case M3D_SOLVER_LINEAR2: {
      if (!chi500 || !g500) return fail(M3D_EINVAL, "linear2 needs chi500 and g500");
      LAUNCH_S(M3D_STAGE_SOLVE, k_long_char2<T>, grid, block, 0, a, work, psi, irem, esc, chi500, g500, eta_row,
             (const uint8_t *)eta_mask, s->ds[2] / fabs(s->vec[2]));
      return M3D_OK;
    }
    case M3D_SOLVER_QUADRATIC: {
      LAUNCH_S(M3D_STAGE_SOLVE, k_long_char_quadratic<T>, grid, block, 0, a, work, psi, quad_const(s->ds[2], s->vec[2]));
      return M3D_OK;
    }
    case M3D_SOLVER_SHORT_LINEAR:
    case M3D_SOLVER_SHORT_LINEAR2: {
      double xk[4], yk[4], dsup;
      int upo1, upo2;
      set_stencil(s->ds, s->vec, xk, yk, &upo1, &upo2, &dsup);
      {
        // set_stencil places the upwind point between the two inner nodes of the
        // 4x4 stencil only when it lies within one cell horizontally; beyond
        // that the cubic kernel extrapolates and the sweep diverges
        const double wt1 = -s->vec[0] / s->ds[0] * dsup, wt2 = -s->vec[1] / s->ds[1] * dsup;
        if (fabs(wt1) > 1.0 || fabs(wt2) > 1.0)
          return fail(M3D_EINVAL,
                      "short characteristics: the upwind point of direction (%g, %g, %g) lies (%g, %g) cells away; "
                      "the stencil reaches one cell (ds_x >= |v_x/v_z| ds_z)",
                      s->vec[0], s->vec[1], s->vec[2], wt1, wt2);
      }
      std::vector<int> tab(4 * (a.nx + a.ny));
      for (int x = 0; x < a.nx; x++)
        for (int ii = 0; ii < 4; ii++) {
          int v = ((ii + 1) + (x + 1) + (upo1 - 2)) % a.nx;
          tab[4 * x + ii] = v < 0 ? v + a.nx : v;
        }
      for (int y = 0; y < a.ny; y++)
        for (int jj = 0; jj < 4; jj++) {
          int v = ((jj + 1) + (y + 1) + (upo2 - 2)) % a.ny;
          tab[4 * a.nx + 4 * y + jj] = v < 0 ? v + a.ny : v;
        }
      void *dtab;
      TRY(scratch(3, sizeof(int) * tab.size(), &dtab));
      CUDA_TRY(cudaMemcpyAsync(dtab, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, g_ctx.stream));
      const int *xt = (const int *)dtab, *yt = xt + 4 * a.nx;
      const float4 kx = make_float4((float)xk[0], (float)xk[1], (float)xk[2], (float)xk[3]);
      const float4 ky = make_float4((float)yk[0], (float)yk[1], (float)yk[2], (float)yk[3]);
      const int zs = a.dir > 0 ? 1 : a.nz;
      if (solver == M3D_SOLVER_SHORT_LINEAR) {
        const T dsup05 = (T)(0.5f * (float)dsup);
        const size_t smem = sizeof(T) * 3 * (SC_TX + 3) * (SC_TY + 3) * SC_TF;
        thread_local bool attr_set[2] = {false, false};
        if (!attr_set[sizeof(T) == 8]) {
          CUDA_TRY(cudaFuncSetAttribute(k_short_char_tile<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
          attr_set[sizeof(T) == 8] = true;
        }
        const int tgrid = ((a.nx + SC_TX - 1) / SC_TX) * ((a.ny + SC_TY - 1) / SC_TY) * ((a.nf + SC_TF - 1) / SC_TF);
        for (int i = 0, z = zs; i < a.nz; i++, z += a.dir)
          LAUNCH_S(M3D_STAGE_SOLVE, k_short_char_tile<T>, tgrid, 256, smem, a, z, work, psi, irem, esc, xt, yt, kx, ky,
                   dsup05);
      } else {
        if (!chi500 || !chi500_up || !g500) return fail(M3D_EINVAL, "linear2 needs chi500, chi500_up and g500");
        const float hx = 2.0f * kx.w + (-kx.x + kx.z), hy = 2.0f * ky.w + (-ky.x + ky.z);
        for (int i = 0, z = zs; i < a.nz; i++, z += a.dir)
          LAUNCH_S(M3D_STAGE_SOLVE, k_short_char2_plane<T>, grid, block, 0, a, z, work, psi, irem, esc, xt, yt, kx, ky, hx, hy, chi500,
                 chi500_up, g500, eta_row, (const uint8_t *)eta_mask, dsup);
      }
      CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
      return M3D_OK;
    }
  }
  return fail(M3D_EINVAL, "unknown solver %d", solver);
}

template <typename T>
int formal_solve_t(int solver, const m3d_slab_t *s, void *work, void *psi, void *irem, void *escape,
                   const float *chi500, const float *chi500_up, const float *g500, const int *eta_row,
                   const unsigned char *eta_mask, const double *rot_ds_code, double rot_bot2pivot,
                   const double *rot_offset, unsigned flags) {
  Staging st(flags);
  const size_t nw = (size_t)s->nf * s->nx * s->ny * (s->nz + 2) * 3;
  const size_t np = (size_t)s->nf * s->nx * s->ny * s->nz;
  const size_t nc = (size_t)s->nx * s->ny * s->nz;
  const SlabArgs a = slab_args(s, flags);
  T *dw, *dp = nullptr, *dir_ = nullptr, *de = nullptr;
  TRY(st.map((T *)work, nw, true, true, &dw));
  if (a.get_psi) TRY(st.map((T *)psi, np, true, true, &dp));
  if (a.split_rates) {
    TRY(st.map((T *)irem, np, true, true, &dir_));
    TRY(st.map((T *)escape, np, true, true, &de));
  }
  const float *c5 = nullptr, *c5u = nullptr, *g5 = nullptr;
  const int *er = nullptr;
  const unsigned char *em = nullptr;
  if (solver == M3D_SOLVER_LINEAR2 || solver == M3D_SOLVER_SHORT_LINEAR2) {
    TRY(st.in(chi500, nc, &c5));
    TRY(st.in(g500, (size_t)s->nx * s->ny, &g5));
    if (solver == M3D_SOLVER_SHORT_LINEAR2) TRY(st.in(chi500_up, nc, &c5u));
    if (eta_row) {
      TRY(st.in(eta_row, nc, &er));
      if (!eta_mask) return fail(M3D_EINVAL, "eta_row without eta_mask");
      int nrows = 0;
      if (st.device()) {
        return fail(M3D_EUNSUPPORTED, "eta flags with device pointers: pass host buffers");
      }
      for (size_t i = 0; i < nc; i++) nrows = eta_row[i] > nrows ? eta_row[i] : nrows;
      TRY(st.in(eta_mask, (size_t)s->nf * (nrows > 0 ? nrows : 1), &em));
    }
  }
  if ((flags & M3D_ROTATE) && solver == M3D_SOLVER_QUADRATIC) {
    if (!rot_ds_code) return fail(M3D_EINVAL, "M3D_ROTATE needs rot_ds_code");
    TRY(rotate_impl<T>(s, dw, rot_ds_code, rot_bot2pivot, rot_offset));
  }
  TRY(solve_impl<T>(solver, s, flags, dw, dp, dir_, de, c5, c5u, g5, er, em));
  return st.finish();
}

template <typename T>
int boundary_t(const m3d_slab_t *s, void *work, int mode, const void *mem, float ds3_code, const float *ghost_r500,
               const float *ghost_temp, const double *nu, unsigned flags) {
  Staging st(flags);
  const size_t plane = (size_t)s->nf * s->nx * s->ny;
  const size_t nw = plane * (s->nz + 2) * 3;
  T *dw;
  const T *dm = nullptr;
  const float *dr = nullptr, *dt = nullptr;
  const double *dnu = nullptr;
  TRY(st.map((T *)work, nw, true, true, &dw));
  if (mode == M3D_BND_MEM) {
    if (!mem) return fail(M3D_EINVAL, "M3D_BND_MEM needs mem");
    TRY(st.in((const T *)mem, plane * 3, &dm));
  } else if (mode == M3D_BND_LTE) {
    if (!ghost_r500 || !ghost_temp || !nu) return fail(M3D_EINVAL, "M3D_BND_LTE needs ghost_r500, ghost_temp, nu");
    TRY(st.in(ghost_r500, (size_t)s->nx * s->ny, &dr));
    TRY(st.in(ghost_temp, (size_t)s->nx * s->ny, &dt));
    TRY(st.in(nu, s->nf, &dnu));
  } else if (mode != M3D_BND_ZERO && mode != M3D_BND_PCHIP) {
    return fail(M3D_EINVAL, "unknown boundary mode %d", mode);
  }
  LAUNCH(k_upstream_boundary<T>, grid_for(plane), 256, 0, s->nf, s->nx, s->ny, s->nz, s->dir, dw, mode, dm,
         pchip_const(ds3_code), dr, dt, dnu);
  return st.finish();
}

}  // namespace

extern "C" {

int m3d_formal_solve(int solver, const m3d_slab_t *slab, void *work, void *psi, void *irem, void *escape,
                     const float *chi500, const float *chi500_up, const float *g500, const int *eta_row,
                     const unsigned char *eta_mask, const double *rot_ds_code, double rot_bot2pivot,
                     const double *rot_offset, unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work) return fail(M3D_EINVAL, "work is NULL");
  if (flags & M3D_FP64)
    return formal_solve_t<double>(solver, slab, work, psi, irem, escape, chi500, chi500_up, g500, eta_row, eta_mask,
                                  rot_ds_code, rot_bot2pivot, rot_offset, flags);
  return formal_solve_t<float>(solver, slab, work, psi, irem, escape, chi500, chi500_up, g500, eta_row, eta_mask,
                               rot_ds_code, rot_bot2pivot, rot_offset, flags);
}

int m3d_long_char_hermite(const m3d_slab_t *slab, float *work, float *psi, const m3d_hermite_t *h,
                          unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work || !h || !h->beta || !h->pe || !h->dpe_dz || !h->dlnt_dz || !h->temp || !h->hknu)
    return fail(M3D_EINVAL, "m3d_long_char_hermite: NULL argument");
  if (slab->nz < 3) return fail(M3D_EINVAL, "m3d_long_char_hermite: needs nz >= 3 (got %d)", slab->nz);
  if (flags & M3D_FP64) return fail(M3D_EUNSUPPORTED, "m3d_long_char_hermite: FP32 only");
  const bool gt = h->ghost_pe != nullptr;
  if (gt && (!h->ghost_dpe_dz || !h->ghost_dlnt_dz || !h->ghost_temp))
    return fail(M3D_EINVAL, "m3d_long_char_hermite: give all four ghost fields or none");
  if (!(h->code_length > 0)) return fail(M3D_EINVAL, "m3d_long_char_hermite: code_length must be > 0");
  const SlabArgs a = slab_args(slab, flags);
  if (a.get_psi && !psi) return fail(M3D_EINVAL, "m3d_long_char_hermite: get_psi without psi");
  const int nf = a.nf, nx = a.nx, ny = a.ny, nz = a.nz;
  const size_t plane = (size_t)nf * nx * ny, cells = (size_t)nx * ny * nz;
  Staging st(flags);
  float *dw, *dp = nullptr;
  TRY(st.map(work, plane * (nz + 2) * 3, true, true, &dw));
  if (a.get_psi) TRY(st.map(psi, plane * nz, true, true, &dp));
  HermArgs K{};
  TRY(st.in(h->beta, plane * nz, &K.beta));
  TRY(st.in(h->pe, cells, &K.pe));
  TRY(st.in(h->dpe_dz, cells, &K.dpe_dz));
  TRY(st.in(h->dlnt_dz, cells, &K.dlnt_dz));
  TRY(st.in(h->temp, cells, &K.temp));
  TRY(st.in(h->hknu, nf, &K.hknu));
  if (gt) {
    TRY(st.in(h->ghost_pe, (size_t)nx * ny, &K.g_pe));
    TRY(st.in(h->ghost_dpe_dz, (size_t)nx * ny, &K.g_dpe_dz));
    TRY(st.in(h->ghost_dlnt_dz, (size_t)nx * ny, &K.g_dlnt_dz));
    TRY(st.in(h->ghost_temp, (size_t)nx * ny, &K.g_temp));
  }
  // the step constants of long_char_hermite's set-up (rt_solvers_mod.f90:1075-1081)
  const float ds = (float)slab->ds[2];
  const float dsup = (float)((double)ds / fabs(slab->vec[2]));
  K.rdsup = 1.0f / dsup;
  K.dsup1 = 0.5f * dsup;
  K.dsup2 = (0.0833333358f * dsup) * dsup;
  K.dtmax = -(float)slab->maser_dtau_max;
  K.Imax = (float)slab->maser_Inu_max;
  K.gfac = (float)((double)a.dir * fabs(slab->vec[2]) / h->code_length);
  K.get_rates = a.get_psi;
  K.ghost_thermo = gt ? 1 : 0;
  LAUNCH_S(M3D_STAGE_SOLVE, k_long_char_hermite, grid_for(plane), 256, 0, K, nf, nx, ny, nz, a.dir, dw, dp);
  return st.finish();
}

int m3d_long_char_hermite2(const m3d_slab_t *slab, float *work, float *psi, const float *pe, const float *dpe_dz,
                           const float *ghost_pe, const float *ghost_dpe_dz, int ghost, double code_length,
                           unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work || !pe || !dpe_dz) return fail(M3D_EINVAL, "m3d_long_char_hermite2: NULL argument");
  if (slab->nz < 2) return fail(M3D_EINVAL, "m3d_long_char_hermite2: needs nz >= 2 (got %d)", slab->nz);
  if (flags & M3D_FP64) return fail(M3D_EUNSUPPORTED, "m3d_long_char_hermite2: FP32 only");
  if (ghost < 0 || ghost > 2) return fail(M3D_EINVAL, "m3d_long_char_hermite2: ghost must be 0, 1 or 2 (got %d)", ghost);
  if (ghost && (!ghost_pe || !ghost_dpe_dz))
    return fail(M3D_EINVAL, "m3d_long_char_hermite2: ghost %d needs ghost_pe and ghost_dpe_dz", ghost);
  if (!(code_length > 0)) return fail(M3D_EINVAL, "m3d_long_char_hermite2: code_length must be > 0");
  const SlabArgs a = slab_args(slab, flags);
  if (a.get_psi && !psi) return fail(M3D_EINVAL, "m3d_long_char_hermite2: get_psi without psi");
  const int nf = a.nf, nx = a.nx, ny = a.ny, nz = a.nz;
  const size_t plane = (size_t)nf * nx * ny, cells = (size_t)nx * ny * nz;
  Staging st(flags);
  float *dw, *dp = nullptr;
  TRY(st.map(work, plane * (nz + 2) * 3, true, true, &dw));
  if (a.get_psi) TRY(st.map(psi, plane * nz, true, true, &dp));
  Herm2Args K{};
  TRY(st.in(pe, cells, &K.pe));
  TRY(st.in(dpe_dz, cells, &K.dpe_dz));
  if (ghost) {
    TRY(st.in(ghost_pe, (size_t)nx * ny, &K.g_pe));
    TRY(st.in(ghost_dpe_dz, (size_t)nx * ny, &K.g_dpe_dz));
  }
  // the step constants of long_char_hermite2's set-up (rt_solvers_mod.f90:1560-1566)
  const float ds = (float)slab->ds[2];
  const float dsup = (float)((double)ds / fabs(slab->vec[2]));
  K.rdsup = 1.0f / dsup;
  K.dsup1 = 0.5f * dsup;
  K.dsup2 = (0.0833333358f * dsup) * dsup;
  K.dtmax = -slab->maser_dtau_max;
  K.Imax = (float)slab->maser_Inu_max;
  K.gfac = (float)((double)a.dir * fabs(slab->vec[2]) / code_length);
  K.get_rates = a.get_psi;
  K.ghost = ghost;
  LAUNCH_S(M3D_STAGE_SOLVE, k_long_char_hermite2, grid_for(plane), 256, 0, K, nf, nx, ny, nz, a.dir, dw, dp);
  return st.finish();
}

int m3d_short_char_hermite(const m3d_slab_t *slab, float *work, float *psi, float *irem, float *escape,
                           const m3d_hermite3d_t *h, unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work || !h || !h->beta || !h->pe || !h->dpe_dx || !h->dpe_dy || !h->dpe_dz || !h->dlnt_dx || !h->dlnt_dy ||
      !h->dlnt_dz || !h->temp || !h->hknu)
    return fail(M3D_EINVAL, "m3d_short_char_hermite: NULL argument");
  if (flags & M3D_FP64) return fail(M3D_EUNSUPPORTED, "m3d_short_char_hermite: FP32 only");
  if (!(h->code_length > 0)) return fail(M3D_EINVAL, "m3d_short_char_hermite: code_length must be > 0");
  const SlabArgs a = slab_args(slab, flags);
  if (a.get_psi && !psi) return fail(M3D_EINVAL, "m3d_short_char_hermite: get_psi without psi");
  if (a.split_rates && (!irem || !escape)) return fail(M3D_EINVAL, "m3d_short_char_hermite: split_rates without irem/escape");
  double xk[4], yk[4], dsup;
  int upo1, upo2;
  set_stencil(slab->ds, slab->vec, xk, yk, &upo1, &upo2, &dsup);
  {
    const double wt1 = -slab->vec[0] / slab->ds[0] * dsup, wt2 = -slab->vec[1] / slab->ds[1] * dsup;
    if (fabs(wt1) > 1.0 || fabs(wt2) > 1.0)
      return fail(M3D_EINVAL,
                  "short characteristics: the upwind point of direction (%g, %g, %g) lies (%g, %g) cells away; "
                  "the stencil reaches one cell (ds_x >= |v_x/v_z| ds_z)",
                  slab->vec[0], slab->vec[1], slab->vec[2], wt1, wt2);
  }
  const int nf = a.nf, nx = a.nx, ny = a.ny, nz = a.nz;
  const size_t plane = (size_t)nf * nx * ny, cells = (size_t)nx * ny * nz;
  Staging st(flags);
  float *dw, *dp = nullptr, *dr = nullptr, *de = nullptr;
  TRY(st.map(work, plane * (nz + 2) * 3, true, true, &dw));
  if (a.get_psi) TRY(st.map(psi, plane * nz, true, true, &dp));
  if (a.split_rates) {
    TRY(st.map(irem, plane * nz, true, true, &dr));
    TRY(st.map(escape, plane * nz, true, true, &de));
  }
  SCHermArgs K{};
  TRY(st.in(h->beta, plane * nz, &K.beta));
  TRY(st.in(h->pe, cells, &K.pe));
  TRY(st.in(h->dpe_dx, cells, &K.dpe_dx));
  TRY(st.in(h->dpe_dy, cells, &K.dpe_dy));
  TRY(st.in(h->dpe_dz, cells, &K.dpe_dz));
  TRY(st.in(h->dlnt_dx, cells, &K.dlnt_dx));
  TRY(st.in(h->dlnt_dy, cells, &K.dlnt_dy));
  TRY(st.in(h->dlnt_dz, cells, &K.dlnt_dz));
  TRY(st.in(h->temp, cells, &K.temp));
  TRY(st.in(h->hknu, nf, &K.hknu));
  std::vector<int> tab(4 * (nx + ny));
  for (int x = 0; x < nx; x++)
    for (int ii = 0; ii < 4; ii++) tab[4 * x + ii] = wrap_host((ii + 1) + (x + 1) + (upo1 - 2), nx);
  for (int y = 0; y < ny; y++)
    for (int jj = 0; jj < 4; jj++) tab[4 * nx + 4 * y + jj] = wrap_host((jj + 1) + (y + 1) + (upo2 - 2), ny);
  void *dtab;
  TRY(scratch(3, sizeof(int) * tab.size(), &dtab));
  CUDA_TRY(cudaMemcpyAsync(dtab, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  K.xt = (const int *)dtab;
  K.yt = K.xt + 4 * nx;
  K.kx = make_float4((float)xk[0], (float)xk[1], (float)xk[2], (float)xk[3]);
  K.ky = make_float4((float)yk[0], (float)yk[1], (float)yk[2], (float)yk[3]);
  // the set-up of short_char_hermite (rt_solvers_mod.f90:1961-1999)
  const double sg = copysign(1.0, slab->vec[2]) * (double)a.dir;
  K.v1 = (float)(slab->vec[0] * sg / h->code_length);
  K.v2 = (float)(slab->vec[1] * sg / h->code_length);
  K.v3 = (float)(slab->vec[2] * sg / h->code_length);
  K.dsup05 = 0.5f * (float)dsup;
  K.rpath = 0.5f / K.dsup05;
  K.dsc2 = (K.dsup05 * K.dsup05) / 3.0f;
  K.dtmaxf = -(float)slab->maser_dtau_max;
  K.dtmax = -slab->maser_dtau_max;
  K.Imax = (float)slab->maser_Inu_max;
  const int zs = a.dir > 0 ? 1 : nz;
  for (int i = 0, z = zs; i < nz; i++, z += a.dir)
    LAUNCH_S(M3D_STAGE_SOLVE, k_short_char_hermite_plane, grid_for(plane), 256, 0, a, K, z, dw, dp, dr, de);
  CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  return st.finish();
}

int m3d_rotate_array(const m3d_slab_t *slab, void *work, const double *ds_code, double bot2pivot,
                     const double *ray_offset, unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work || !ds_code) return fail(M3D_EINVAL, "m3d_rotate_array: NULL work or ds_code");
  const size_t nw = (size_t)slab->nf * slab->nx * slab->ny * (slab->nz + 2) * 3;
  Staging st(flags);
  if (flags & M3D_FP64) {
    double *dw;
    TRY(st.map((double *)work, nw, true, true, &dw));
    TRY(rotate_impl<double>(slab, dw, ds_code, bot2pivot, ray_offset));
  } else {
    float *dw;
    TRY(st.map((float *)work, nw, true, true, &dw));
    TRY(rotate_impl<float>(slab, dw, ds_code, bot2pivot, ray_offset));
  }
  return st.finish();
}

int m3d_upstream_boundary(const m3d_slab_t *slab, void *work, int mode, const void *mem, float ds3_code,
                          const float *ghost_r500, const float *ghost_temp, const double *nu, unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work) return fail(M3D_EINVAL, "work is NULL");
  if (flags & M3D_FP64) return boundary_t<double>(slab, work, mode, mem, ds3_code, ghost_r500, ghost_temp, nu, flags);
  return boundary_t<float>(slab, work, mode, mem, ds3_code, ghost_r500, ghost_temp, nu, flags);
}

// ---------------------------------------------------------------------------
// LTE synthesis output pass of one window
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

// The atmosphere, line lists and window of the LTE pass on the device
struct SynthIn {
  AtmosDev A;
  std::vector<SpeciesDev> sp;
  bool reach = false;
  unsigned *d_vmax = nullptr;
  std::vector<int *> d_sel, d_nsel;
  GridArgs G;
  const double *dnu = nullptr, *dllam = nullptr;
  int nf = 0;
  size_t ncell = 0;
  // a batch of nwin windows of nf frequencies (nu, llam of nwin nf), each with its grid,
  // for nray directions d_vr (3 each) in one launch
  int nwin = 1;
  const GridArgs *d_Gw = nullptr;
  int nray = 1;
  const double *d_vr = nullptr;
};

int stage_synthesis(Staging &st, const m3d_atmos_t *atm, int nf, const double *nu, const double *llam, bool fp64,
                    const char *who, SynthIn *in) {
  const int nx = atm->nx, ny = atm->ny, nz = atm->nz;
  const size_t ncell = (size_t)nx * ny * nz;
  if (ncell > (size_t)INT_MAX / 2) return fail(M3D_EUNSUPPORTED, "%s: %zu cells", who, ncell);
  in->nf = nf;
  in->ncell = ncell;
  AtmosDev &A = in->A;
  A.ncell = (int)ncell;
  TRY(st.in(atm->temp, ncell, &A.temp)); TRY(st.in(atm->chi_c, ncell, &A.chi_c));
  TRY(st.in(atm->vx, ncell, &A.vx)); TRY(st.in(atm->vy, ncell, &A.vy)); TRY(st.in(atm->vz, ncell, &A.vz));
  TRY(st.in(atm->e_kT, ncell, &A.e_kT)); TRY(st.in(atm->ne, ncell, &A.ne));
  TRY(st.in(atm->tothi, ncell, &A.tothi)); TRY(st.in(atm->stark_pe, ncell, &A.stark_pe));
  if (!A.temp || !A.chi_c || !A.vx || !A.vy || !A.vz || !A.e_kT || !A.ne || !A.tothi || !A.stark_pe)
    return fail(M3D_EINVAL, "%s: NULL atmosphere field", who);
  A.maser_chi_floor = (float)atm->maser_chi_floor;
  A.nspecies = atm->nspecies;
  in->sp.assign(atm->nspecies > 0 ? atm->nspecies : 1, SpeciesDev{});
  auto &sp = in->sp;
  size_t nsel_all = 0;
  for (int k = 0; k < atm->nspecies; k++) {
    TRY(stage_linelist(st, &atm->species[k].ll, &sp[k].L));
    TRY(st.in(atm->species[k].inv_df, ncell, &sp[k].inv_df));
    TRY(st.in(atm->species[k].vbar2, ncell, &sp[k].vbar2));
    TRY(st.in(atm->species[k].lnbase, ncell, &sp[k].lnbase));
    if (sp[k].L.reach_in) in->reach = true;
    nsel_all += (size_t)sp[k].L.nline + 8;
  }
  if (in->reach && fp64) return fail(M3D_EUNSUPPORTED, "%s: reach_in with the FP64 path", who);
  // select_lines per ray: a vmax word, then per species its count and its list
  in->d_sel.assign(sp.size(), nullptr);
  in->d_nsel.assign(sp.size(), nullptr);
  if (in->reach) {
    for (int k = 0; k < atm->nspecies; k++)
      if (!sp[k].L.reach_in) return fail(M3D_EINVAL, "%s: reach_in given for some species only", who);
    void *sbuf = nullptr;
    TRY(scratch(21, sizeof(int) * (nsel_all + 8), &sbuf));
    in->d_vmax = (unsigned *)sbuf;
    int *p = (int *)sbuf + 8;
    for (int k = 0; k < atm->nspecies; k++) {
      in->d_nsel[k] = p;
      in->d_sel[k] = p + 8;
      p += sp[k].L.nline + 8;
      sp[k].L.sel = in->d_sel[k];
      sp[k].L.nsel = in->d_nsel[k];
    }
  }
  void *dsp;
  TRY(scratch(4, sizeof(SpeciesDev) * sp.size(), &dsp));
  CUDA_TRY(cudaMemcpyAsync(dsp, sp.data(), sizeof(SpeciesDev) * sp.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  A.species = (const SpeciesDev *)dsp;
  TRY(st.in(nu, nf, &in->dnu));
  TRY(st.in(llam, nf, &in->dllam));
  in->G = grid_args(nf, llam, in->dllam, st.device(), (float)atm->tol, 0.0f);
  if (!(in->G.dllam > 0)) return fail(M3D_EINVAL, "%s: log(lambda) grid must be ascending", who);
  return M3D_OK;
}

// Line opacity + transfer units of every cell for direction v: (chi, S) of the
// window, frequency fastest per cell.  FP32: the lane-per-cell kernel for windows of
// 32 frequencies, the warp-per-cell kernel otherwise; FP64: the plain FP64 kernel.
int launch_opacity(SynthIn &in, const double *v, bool fp64, void *dchi, void *dS) {
  const int nf = in.nf;
  const size_t ncell = in.ncell;
  const int block = 256, warps = block / 32;
  const bool batch = in.nwin > 1;
  if (fp64) {
    int grid = (int)((ncell * in.nwin * (batch ? in.nray : 1) + block - 1) / block);
    if (grid > 148 * 8) grid = 148 * 8;
    if (batch)
      LAUNCH_S(M3D_STAGE_OPACITY, (k_lte_opacity_units_f64<32, true>), grid, block, 0, in.A, in.G, in.dnu, 0.0, 0.0,
               0.0, (double *)dchi, (double *)dS, (const double2 *)g_ctx.d_tab64, in.d_Gw, in.nwin, in.d_vr, in.nray);
    else if (nf == 32)
      LAUNCH_S(M3D_STAGE_OPACITY, k_lte_opacity_units_f64<32>, grid, block, 0, in.A, in.G, in.dnu, v[0], v[1], v[2],
               (double *)dchi, (double *)dS, (const double2 *)g_ctx.d_tab64, (const GridArgs *)nullptr, 1,
               (const double *)nullptr, 1);
    else
      LAUNCH_S(M3D_STAGE_OPACITY, k_lte_opacity_units_f64<0>, grid, block, 0, in.A, in.G, in.dnu, v[0], v[1], v[2],
               (double *)dchi, (double *)dS, (const double2 *)g_ctx.d_tab64, (const GridArgs *)nullptr, 1,
               (const double *)nullptr, 1);
    return M3D_OK;
  }
  const bool lane32 = nf == 32;
  const size_t smem_op = lane32 ? 2 * QLG_NTAB * sizeof(float)
                                : (2 * QLG_NTAB + (size_t)warps * 4 * nf) * sizeof(float);
  {
    thread_local size_t attr[2] = {0, 0};
    const int which = lane32 ? 1 : 0;
    if (attr[which] < smem_op) {
      if (lane32) {
        CUDA_TRY(cudaFuncSetAttribute((const void *)k_lte_opacity_units_lane<32, float, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_op));
        CUDA_TRY(cudaFuncSetAttribute((const void *)k_lte_opacity_units_lane<32, float, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_op));
        CUDA_TRY(cudaFuncSetAttribute((const void *)k_lte_opacity_units_lane<32, float, false, false, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_op));
      } else {
        CUDA_TRY(cudaFuncSetAttribute((const void *)k_lte_opacity_units<float>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_op));
      }
      attr[which] = smem_op;
    }
  }
  if (in.reach) {
    CUDA_TRY(cudaMemsetAsync(in.d_vmax, 0, sizeof(unsigned), g_ctx.stream));
    LAUNCH(k_vproj_absmax, grid_for(ncell), 256, 0, in.A, v[0], v[1], v[2], in.d_vmax);
    for (int k = 0; k < in.A.nspecies; k++)
      LAUNCH(k_select_lines, 1, 32, 0, in.sp[k].L, in.dllam, nf, (const unsigned *)in.d_vmax, in.d_sel[k],
             in.d_nsel[k]);
  }
  if (lane32) {
    // lane kernel: one warp per 32 cells (of one window), grid-stride over warps.  One
    // block of 24 warps per SM: the QLG tables are staged once per SM (72 KB), where
    // three blocks of 8 warps (the same occupancy) held three copies and left L1 almost
    // no room for the line list and the cells' fields; 3.55 -> 4.08 Gpt*nu*ray/s on the
    // 240^3 configuration
    const size_t nvc = (ncell + 31) / 32 * 32 * (size_t)in.nwin * (batch ? in.nray : 1);
    const int lblock = 768;
    int lgrid = (int)((nvc + lblock - 1) / lblock);
    if (lgrid > 148 * 8) lgrid = 148 * 8;
    if (batch)
      LAUNCH_S(M3D_STAGE_OPACITY, (k_lte_opacity_units_lane<32, float, false, false, true>), lgrid, lblock, smem_op,
               in.A, in.G, in.dnu, 0.0, 0.0, 0.0, (float *)dchi, (float *)dS, g_ctx.d_tab, in.d_Gw, in.nwin, in.d_vr,
               in.nray);
    else if (in.reach)
      LAUNCH_S(M3D_STAGE_OPACITY, (k_lte_opacity_units_lane<32, float, true>), lgrid, lblock, smem_op, in.A, in.G,
               in.dnu, v[0], v[1], v[2], (float *)dchi, (float *)dS, g_ctx.d_tab, (const GridArgs *)nullptr, 1,
               (const double *)nullptr, 1);
    else
      LAUNCH_S(M3D_STAGE_OPACITY, (k_lte_opacity_units_lane<32, float, false>), lgrid, lblock, smem_op, in.A, in.G,
               in.dnu, v[0], v[1], v[2], (float *)dchi, (float *)dS, g_ctx.d_tab, (const GridArgs *)nullptr, 1,
               (const double *)nullptr, 1);
  } else {
    int ogrid = (int)((ncell + warps - 1) / warps);
    if (ogrid > 148 * 16) ogrid = 148 * 16;
    LAUNCH_S(M3D_STAGE_OPACITY, k_lte_opacity_units<float>, ogrid, block, smem_op, in.A, in.G, in.dnu, v[0], v[1],
             v[2], (float *)dchi, (float *)dS, g_ctx.d_tab);
  }
  return M3D_OK;
}

int check_synthesis_args(const m3d_atmos_t *atm, int nf, const char *who) {
  if (nf < 2) return fail(M3D_EINVAL, "%s: need nf >= 2", who);
  if (nf > 1024) return fail(M3D_EUNSUPPORTED, "%s: nf = %d > 1024 per window", who, nf);
  if (atm->nx < 1 || atm->ny < 1 || atm->nz < 1) return fail(M3D_EINVAL, "%s: bad atmosphere shape", who);
  return M3D_OK;
}

int lte_synthesis_impl(const m3d_atmos_t *atm, int nwin, int nf_win, const double *nu, const double *llam, int nray,
                       const double *vec, const double *wmu, void *i_top, float *ie, float *flux, unsigned flags,
                       const char *who);

}  // namespace

extern "C" {

int m3d_lte_transfer_units(const m3d_atmos_t *atm, int nf, const double *nu, const double *llam, const double *vec,
                           void *chi, void *S, unsigned flags) {
  TRY(need_init());
  if (!atm || !nu || !llam || !vec || !chi || !S) return fail(M3D_EINVAL, "m3d_lte_transfer_units: NULL argument");
  TRY(check_synthesis_args(atm, nf, "m3d_lte_transfer_units"));
  const bool fp64 = flags & M3D_FP64;
  Staging st(flags);
  SynthIn in;
  TRY(stage_synthesis(st, atm, nf, nu, llam, fp64, "m3d_lte_transfer_units", &in));
  const size_t n = (size_t)nf * in.ncell;
  void *dchi, *dS;
  if (fp64) {
    double *a, *b;
    TRY(st.map((double *)chi, n, false, true, &a));
    TRY(st.map((double *)S, n, false, true, &b));
    dchi = a; dS = b;
  } else {
    float *a, *b;
    TRY(st.map((float *)chi, n, false, true, &a));
    TRY(st.map((float *)S, n, false, true, &b));
    dchi = a; dS = b;
  }
  TRY(launch_opacity(in, vec, fp64, dchi, dS));
  return st.finish();
}

int m3d_lte_synthesis(const m3d_atmos_t *atm, int nf, const double *nu, const double *llam, int nray,
                      const double *vec, const double *wmu, void *i_top, float *ie, float *flux, unsigned flags) {
  return lte_synthesis_impl(atm, 1, nf, nu, llam, nray, vec, wmu, i_top, ie, flux, flags, "m3d_lte_synthesis");
}

int m3d_lte_synthesis_windows(const m3d_atmos_t *atm, int nwin, int nf, const double *nu, const double *llam,
                              int nray, const double *vec, const double *wmu, void *i_top, float *ie, float *flux,
                              unsigned flags) {
  return lte_synthesis_impl(atm, nwin, nf, nu, llam, nray, vec, wmu, i_top, ie, flux, flags,
                            "m3d_lte_synthesis_windows");
}

}  // extern "C"

namespace {

// m3d_lte_synthesis for nwin consecutive windows of nf frequencies at once (nwin = 1:
// one window).  The windows' transfer units are laid out as the rows of one window
// of nwin nf frequencies, which the sweep, the reduction and the flux take as such:
// each frequency's arithmetic is the single window's.
int lte_synthesis_impl(const m3d_atmos_t *atm, int nwin, int nf_win, const double *nu, const double *llam, int nray,
                       const double *vec, const double *wmu, void *i_top, float *ie, float *flux, unsigned flags,
                       const char *who) {
  TRY(need_init());
  if (!atm || !nu || !llam || !vec || !wmu || !ie || !flux) return fail(M3D_EINVAL, "%s: NULL argument", who);
  if (nray < 1) return fail(M3D_EINVAL, "%s: need nray >= 1", who);
  if (nwin < 1) return fail(M3D_EINVAL, "%s: need nwin >= 1", who);
  TRY(check_synthesis_args(atm, nf_win, who));
  if (nwin > 1 && nf_win != 32) return fail(M3D_EUNSUPPORTED, "%s: window batches of nf = 32 only", who);
  if ((size_t)nwin * nf_win > (size_t)INT_MAX / 2) return fail(M3D_EUNSUPPORTED, "%s: %d windows", who, nwin);
  const int nf = nwin * nf_win;   // the frequencies of all windows, one after the other
  const int nx = atm->nx, ny = atm->ny, nz = atm->nz;
  if (nz < 2 || atm->nslab < 1 || !atm->slab_nz) return fail(M3D_EINVAL, "m3d_lte_synthesis: bad atmosphere shape");
  std::vector<int> z0(atm->nslab + 1, 0);
  for (int s = 0; s < atm->nslab; s++) {
    if (atm->slab_nz[s] < 2) return fail(M3D_EINVAL, "slab %d has %d < 2 planes", s, atm->slab_nz[s]);
    z0[s + 1] = z0[s] + atm->slab_nz[s];
  }
  if (z0[atm->nslab] != nz) return fail(M3D_EINVAL, "slab planes sum to %d, not nz = %d", z0[atm->nslab], nz);
  for (int r = 0; r < nray; r++)
    if (!(vec[3 * r + 2] > 0)) return fail(M3D_EINVAL, "ray %d is not upward (vec(3) <= 0)", r);
  const bool fp64 = flags & M3D_FP64;
  const size_t ncol = (size_t)nx * ny;
  const size_t plane = (size_t)nf * ncol;

  Staging st(flags);
  SynthIn in;
  TRY(stage_synthesis(st, atm, nf, nu, llam, fp64, who, &in));
  const double *dnu = in.dnu;
  if (nwin > 1) {
    // every window's grid, as a call for that window alone forms it
    if (in.reach) return fail(M3D_EUNSUPPORTED, "%s: reach_in with window batches", who);
    if ((in.ncell + 31) / 32 * 32 * (size_t)nwin > (size_t)INT_MAX)
      return fail(M3D_EUNSUPPORTED, "%s: %zu cells x %d windows", who, in.ncell, nwin);
    std::vector<double> hl((size_t)nf);
    if (st.device()) {
      CUDA_TRY(cudaMemcpyAsync(hl.data(), llam, sizeof(double) * hl.size(), cudaMemcpyDeviceToHost, g_ctx.stream));
      CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
    } else {
      memcpy(hl.data(), llam, sizeof(double) * hl.size());
    }
    std::vector<GridArgs> gw(nwin);
    for (int w = 0; w < nwin; w++) {
      gw[w] = grid_args(nf_win, hl.data() + (size_t)nf_win * w, in.dllam + (size_t)nf_win * w, false,
                        (float)atm->tol, 0.0f);
      if (!(gw[w].dllam > 0)) return fail(M3D_EINVAL, "%s: window %d: log(lambda) must be ascending", who, w);
    }
    void *dgw, *dvr;
    TRY(scratch(25, sizeof(GridArgs) * gw.size(), &dgw));
    CUDA_TRY(cudaMemcpyAsync(dgw, gw.data(), sizeof(GridArgs) * gw.size(), cudaMemcpyHostToDevice, g_ctx.stream));
    TRY(scratch(26, sizeof(double) * 3 * nray, &dvr));
    CUDA_TRY(cudaMemcpyAsync(dvr, vec, sizeof(double) * 3 * nray, cudaMemcpyHostToDevice, g_ctx.stream));
    in.nf = nf_win;
    in.nwin = nwin;
    in.d_Gw = (const GridArgs *)dgw;
    in.nray = nray;
    in.d_vr = (const double *)dvr;
  }
  // a batch holds every ray's transfer units at once (the opacity of all of them is
  // one launch); a single window one ray's
  const size_t nray_units = nwin > 1 ? (size_t)nray : 1;

  // rotation table of every global plane, per ray; slab starts
  // A single column is a plane-parallel atmosphere: radiative_transfer applies no
  // rotate_array there (rt_patch_mod.f90:1670), so its planes keep identity weights.
  const bool one_d = nx == 1 && ny == 1;
  std::vector<RotPlane> rot((size_t)nray * nz);
  for (int r = 0; r < nray; r++)
    for (int s = 0; s < atm->nslab; s++) {
      const float bottom = (float)((double)z0[s] * atm->ds_code[2]);
      const double b2p = atm->pivot_z - (double)bottom;
      RotPlane *out = rot.data() + (size_t)r * nz + z0[s];
      if (one_d) {
        for (int z = 0; z < atm->slab_nz[s]; z++) out[z] = RotPlane{0, 0, 1.0f, 0.0f, 0.0f, 0.0f};
      } else {
        rot_planes(vec + 3 * r, atm->ds_code, b2p, atm->ray_offset, atm->slab_nz[s], out);
      }
    }
  // the fused sweep takes the periodic offsets reduced to [0, n)
  std::vector<RotCol> rotc(rot.size());
  for (size_t i = 0; i < rot.size(); i++) {
    int ux = rot[i].up1 % nx, uy = rot[i].up2 % ny;
    rotc[i] = RotCol{ux < 0 ? ux + nx : ux, uy < 0 ? uy + ny : uy, rot[i].a, rot[i].b, rot[i].c, rot[i].d};
  }
  void *drot, *dz0;
  TRY(scratch(5, sizeof(RotCol) * rotc.size(), &drot));
  TRY(scratch(6, sizeof(int) * z0.size(), &dz0));
  CUDA_TRY(cudaMemcpyAsync(drot, rotc.data(), sizeof(RotCol) * rotc.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  CUDA_TRY(cudaMemcpyAsync(dz0, z0.data(), sizeof(int) * z0.size(), cudaMemcpyHostToDevice, g_ctx.stream));

  // transfer units of the whole column (one ray at a time) and the emergent planes
  const size_t esz = fp64 ? sizeof(double) : sizeof(float);
  void *dchi, *dS, *dtop;
  TRY(scratch(7, esz * plane * nz * nray_units, &dchi));
  TRY(scratch(8, esz * plane * nz * nray_units, &dS));
  void *dtop_user = nullptr;
  if (i_top) {
    if (fp64) { double *p; TRY(st.map((double *)i_top, plane * nray, false, true, &p)); dtop_user = p; }
    else { float *p; TRY(st.map((float *)i_top, plane * nray, false, true, &p)); dtop_user = p; }
    dtop = dtop_user;
  } else {
    TRY(scratch(9, esz * plane * nray, &dtop));
  }
  float *die;
  TRY(st.map(ie, (size_t)nf * nray, false, true, &die));

  const float dtmax = -(float)atm->maser_dtau_max, Imax = (float)atm->maser_Inu_max;
  const PchipConst pc = pchip_const((float)atm->ds_code[2]);

  // partial sums of the intensity reduction
  const int kParts = 148;
  void *dpart;
  TRY(scratch(12, sizeof(double) * kParts * nf, &dpart));

  // FP64 plain path buffers
  void *dwork = nullptr, *dmem = nullptr;
  int maxn = 0;
  for (int s = 0; s < atm->nslab; s++) maxn = atm->slab_nz[s] > maxn ? atm->slab_nz[s] : maxn;
  if (fp64) {
    TRY(scratch(10, sizeof(double) * plane * (maxn + 2) * 3, &dwork));
    TRY(scratch(11, sizeof(double) * plane * 3, &dmem));
  }

  // a batch's opacity: every ray and window in one launch
  if (nwin > 1) TRY(launch_opacity(in, vec, fp64, dchi, dS));
  for (int r = 0; r < nray; r++) {
    const double *v = vec + 3 * r;
    if (nwin == 1) TRY(launch_opacity(in, v, fp64, dchi, dS));
    // this ray's transfer units
    const size_t ru = nwin > 1 ? plane * nz * (size_t)r : 0;
    const void *rchi = (const char *)dchi + esz * ru, *rS = (const char *)dS + esz * ru;
    if (!fp64) {
      const QuadConst qc = quad_const(atm->ds_cm[2], v[2]);
      if (nf % 2 == 0) {
        // frequency pairs: 8-byte taps, the ray's rotation weights in shared memory
        const size_t pairs = plane / 2;
        LAUNCH_S(M3D_STAGE_SOLVE, k_quad_rot_column2, (int)((pairs + 255) / 256), 256, sizeof(RotCol) * nz, nf, nx, ny,
                 nz, (const float *)rchi, (const float *)rS, (const RotCol *)drot + (size_t)r * nz, (const int *)dz0,
                 atm->nslab, qc, pc, dtmax, Imax, (float *)dtop + plane * r);
      } else {
        LAUNCH_S(M3D_STAGE_SOLVE, k_quad_rot_column, (int)((plane + 255) / 256), 256, 0, nf, nx, ny, nz,
                 (const float *)rchi, (const float *)rS, (const RotCol *)drot + (size_t)r * nz, (const int *)dz0,
                 atm->nslab, qc, pc, dtmax, Imax, (float *)dtop + plane * r);
      }
      LAUNCH_S(M3D_STAGE_REDUCE, k_save_partial<float>, dim3((nf + 31) / 32, kParts), dim3(32, 8), 0, nf, (int)ncol,
               dnu, (const float *)dtop + plane * r, (double *)dpart);
      LAUNCH_S(M3D_STAGE_REDUCE, k_save_final, (nf + 127) / 128, 128, 0, nf, (int)ncol, kParts, (const double *)dpart,
               die + (size_t)nf * r);
    } else {
      for (int s = 0; s < atm->nslab; s++) {
        const int n = atm->slab_nz[s];
        m3d_slab_t sl;
        memset(&sl, 0, sizeof sl);
        sl.nf = nf; sl.nx = nx; sl.ny = ny; sl.nz = n; sl.dir = 1;
        for (int i = 0; i < 3; i++) { sl.ds[i] = atm->ds_cm[i]; sl.vec[i] = v[i]; }
        sl.maser_dtau_max = atm->maser_dtau_max;
        sl.maser_Inu_max = atm->maser_Inu_max;
        double *w = (double *)dwork;
        LAUNCH(k_slab_in, grid_for(plane * n), 256, 0, plane, n, (const double *)rchi + plane * z0[s],
               (const double *)rS + plane * z0[s], w, n);
        LAUNCH(k_upstream_boundary<double>, grid_for(plane), 256, 0, nf, nx, ny, n, 1, w, s == 0 ? M3D_BND_PCHIP : M3D_BND_MEM,
               (const double *)dmem, pc, (const float *)nullptr, (const float *)nullptr, (const double *)nullptr);
        const float bottom = (float)((double)z0[s] * atm->ds_code[2]);
        if (!one_d) TRY(rotate_impl<double>(&sl, w, atm->ds_code, atm->pivot_z - (double)bottom, atm->ray_offset));
        TRY(solve_impl<double>(M3D_SOLVER_QUADRATIC, &sl, 0, w, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                               nullptr, nullptr));
        // exit plane -> mem (chi, S, I at plane n)
        for (int k = 0; k < 3; k++)
          CUDA_TRY(cudaMemcpyAsync((double *)dmem + plane * k, w + plane * ((size_t)n + (size_t)k * (n + 2)),
                                   sizeof(double) * plane, cudaMemcpyDeviceToDevice, g_ctx.stream));
      }
      CUDA_TRY(cudaMemcpyAsync((double *)dtop + plane * r, (double *)dmem + 2 * plane, sizeof(double) * plane,
                               cudaMemcpyDeviceToDevice, g_ctx.stream));
      LAUNCH_S(M3D_STAGE_REDUCE, k_save_partial<double>, dim3((nf + 31) / 32, kParts), dim3(32, 8), 0, nf,
               (int)ncol, dnu, (const double *)dtop + plane * r, (double *)dpart);
      LAUNCH_S(M3D_STAGE_REDUCE, k_save_final, (nf + 127) / 128, 128, 0, nf, (int)ncol, kParts, (const double *)dpart,
               die + (size_t)nf * r);
    }
  }
  TRY(st.finish());
  // flux = 2 pi sum_mu wmu ie (rt_patch_mod.f90:4193-4200), ie now on the host or device
  std::vector<float> hie((size_t)nf * nray);
  if (st.device()) {
    CUDA_TRY(cudaMemcpyAsync(hie.data(), ie, sizeof(float) * hie.size(), cudaMemcpyDeviceToHost, g_ctx.stream));
    CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  } else {
    memcpy(hie.data(), ie, sizeof(float) * hie.size());
  }
  std::vector<float> hflux(nf, 0.0f);
  for (int r = 0; r < nray; r++) {
    const float w = (float)(2.0 * 3.14159265359 * wmu[r]);
    for (int f = 0; f < nf; f++) hflux[f] = fmaf(w, hie[(size_t)f + (size_t)nf * r], hflux[f]);
  }
  if (st.device()) {
    CUDA_TRY(cudaMemcpyAsync(flux, hflux.data(), sizeof(float) * nf, cudaMemcpyHostToDevice, g_ctx.stream));
    CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  } else {
    memcpy(flux, hflux.data(), sizeof(float) * nf);
  }
  return M3D_OK;
}

}  // namespace

#include "m3d_stateq_api.inc"
#include "m3d_nlte_api.inc"
#include "m3d_continuum_api.inc"
#include "m3d_aux_api.inc"
#include "m3d_columns_api.inc"
#include "m3d_optab_api.inc"
#include "m3d_hprof_api.inc"
#include "m3d_io_api.inc"
#include "m3d_adjoint_api.inc"
#include "m3d_hop_api.inc"

// ===========================================================================
// rotate_array without any allocation.
//
// Some callers cannot let the library allocate device memory: a host program
// that hands all device memory to its own pool (PyTorch's caching allocator, a
// preallocated arena) leaves nothing for cudaMalloc, and a program whose other
// streams must not stall cannot afford the device-wide synchronisation that
// cudaMalloc/cudaFree imply.  This entry point therefore takes its scratch from a
// fixed array in the library's own device image, M3D_NOALLOC_SCRATCH_BYTES
// (8 MiB) large, which every GPU that loads the library holds until the process
// exits.  It rotates one plane at a time through that array, so the limit is one
// plane, nf*nx*ny values.  The array is one per device, shared by every call and
// every host thread's context: calls that overlap on the GPU race on it, so the
// caller serialises them (one stream, or events between streams).
// ===========================================================================
namespace {

constexpr size_t M3D_NOALLOC_SCRATCH_BYTES = (size_t)8 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[M3D_NOALLOC_SCRATCH_BYTES];
// The device address of g_noalloc_scratch on the context's device.  The lookup
// allocates nothing and is repeated on every call, so no address outlives a
// device reset; the context's device is made current for it (and the caller's
// current device restored), since the launches go to that device's stream.
int noalloc_scratch(void **out) {
  int cur = 0;
  CUDA_TRY(cudaGetDevice(&cur));
  if (cur != g_ctx.device) CUDA_TRY(cudaSetDevice(g_ctx.device));
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (cur != g_ctx.device) CUDA_TRY(cudaSetDevice(cur));
  if (e != cudaSuccess) return fail(M3D_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
  *out = p;
  return M3D_OK;
}

// one plane of rotate_array into dst, the weights passed by value
template <typename T>
__global__ void k_rotate_one_plane(int nf, int nx, int ny, const T *src, T *dst, RotPlane r) {
  const size_t plane = (size_t)nf * nx * ny;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < plane; g += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(g % nf), x = (int)((g / nf) % nx), y = (int)(g / ((size_t)nf * nx));
    const int x1 = wrap(x + r.up1, nx), x2 = wrap(x + r.up1 + 1, nx);
    const int y1 = wrap(y + r.up2, ny), y2 = wrap(y + r.up2 + 1, ny);
    T v = (T)r.a * src[(size_t)f + (size_t)nf * ((size_t)x1 + (size_t)nx * y1)];
    v = fma_t((T)r.b, src[(size_t)f + (size_t)nf * ((size_t)x2 + (size_t)nx * y1)], v);
    v = fma_t((T)r.c, src[(size_t)f + (size_t)nf * ((size_t)x1 + (size_t)nx * y2)], v);
    v = fma_t((T)r.d, src[(size_t)f + (size_t)nf * ((size_t)x2 + (size_t)nx * y2)], v);
    dst[g] = v;
  }
}

template <typename T>
int rotate_noalloc_t(const m3d_slab_t *s, T *dwork, const double *ds_code, double bot2pivot,
                     const double *ray_offset) {
  const size_t plane = (size_t)s->nf * s->nx * s->ny;
  if (plane * sizeof(T) > M3D_NOALLOC_SCRATCH_BYTES)
    return fail(M3D_EINVAL, "m3d_rotate_array_noalloc: a plane of %zu values (%zu bytes) exceeds the %zu-byte scratch",
                plane, plane * sizeof(T), M3D_NOALLOC_SCRATCH_BYTES);
  void *tmp = nullptr;
  TRY(noalloc_scratch(&tmp));
  const double off0[2] = {0.0, 0.0};
  const double *off = ray_offset ? ray_offset : off0;
  for (int k = 0; k < 2; k++)
    for (int z = 1; z <= s->nz; z++) {
      T *p = dwork + plane * ((size_t)z + (size_t)k * (s->nz + 2));
      LAUNCH(k_rotate_one_plane<T>, grid_for(plane), 256, 0, s->nf, s->nx, s->ny, (const T *)p, (T *)tmp,
             rot_plane_at(s->vec, ds_code, bot2pivot, off, z));
      CUDA_TRY(cudaMemcpyAsync(p, tmp, sizeof(T) * plane, cudaMemcpyDeviceToDevice, g_ctx.stream));
    }
  return M3D_OK;
}

}  // namespace

extern "C" int m3d_rotate_array_noalloc(const m3d_slab_t *slab, void *work, const double *ds_code, double bot2pivot,
                                        const double *ray_offset, unsigned flags) {
  TRY(need_init());
  TRY(check_slab(slab));
  if (!work || !ds_code) return fail(M3D_EINVAL, "m3d_rotate_array_noalloc: NULL work or ds_code");
  if (!(flags & M3D_DEVICE_PTRS))
    return fail(M3D_EINVAL, "m3d_rotate_array_noalloc: work must be a device pointer (M3D_DEVICE_PTRS); "
                            "staging host buffers would allocate");
  if (flags & M3D_FP64) return rotate_noalloc_t<double>(slab, (double *)work, ds_code, bot2pivot, ray_offset);
  return rotate_noalloc_t<float>(slab, (float *)work, ds_code, bot2pivot, ray_offset);
}

// ---- self-check of the opacity kernels' reciprocal ------------------------------
namespace m3d {
// every float with bit pattern in [lo, hi): rcp_markstein against __frcp_rn
__global__ void k_rcp_check(unsigned lo, unsigned hi, unsigned long long *count, unsigned *first) {
  const unsigned long long n = (unsigned long long)hi - lo;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned b = lo + (unsigned)t;
    const float d = __uint_as_float(b);
    if (__float_as_uint(rcp_markstein(d)) != __float_as_uint(__frcp_rn(d))) {
      atomicAdd(count, 1ull);
      atomicMin(first, b);
    }
  }
}
}  // namespace m3d

extern "C" int m3d_rcp_check(unsigned lo_bits, unsigned hi_bits, unsigned long long *mismatches,
                             unsigned *first_bits) {
  using namespace m3d;
  TRY(need_init());
  if (!mismatches || !first_bits) return fail(M3D_EINVAL, "m3d_rcp_check: NULL outputs");
  if (hi_bits < lo_bits) return fail(M3D_EINVAL, "m3d_rcp_check: hi_bits < lo_bits");
  void *sp = nullptr;
  TRY(scratch(24, 16, &sp));
  unsigned long long *dc = (unsigned long long *)sp;
  unsigned *df = (unsigned *)((char *)sp + 8);
  const unsigned init_first = 0xffffffffu;
  CUDA_TRY(cudaMemsetAsync(dc, 0, 8, g_ctx.stream));
  CUDA_TRY(cudaMemcpyAsync(df, &init_first, 4, cudaMemcpyHostToDevice, g_ctx.stream));
  LAUNCH(k_rcp_check, sm_count() * 16, 256, 0, lo_bits, hi_bits, dc, df);
  CUDA_TRY(cudaMemcpyAsync(mismatches, dc, 8, cudaMemcpyDeviceToHost, g_ctx.stream));
  CUDA_TRY(cudaMemcpyAsync(first_bits, df, 4, cudaMemcpyDeviceToHost, g_ctx.stream));
  CUDA_TRY(cudaStreamSynchronize(g_ctx.stream));
  return M3D_OK;
}

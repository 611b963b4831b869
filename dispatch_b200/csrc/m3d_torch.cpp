// torch.ops.m3d: the library's entry points as PyTorch operators over the same C ABI
// (include/m3dgpu.h), for callers that hold their data in torch CUDA tensors -- the
// role tumult's cffi binding of libhop plays for HOP (HOP/hopacity/core.py:142-170).
//
// Every operator takes CUDA tensors, runs on the calling thread's library context
// (m3d_init on the tensors' device the first time), orders its work on torch's
// current stream (m3d_set_stream), and raises the library's error message.  The
// atmosphere of the LTE pass travels as two tensor lists and two number lists:
//   cells   temp, chi_c, vx, vy, vz, e_kT, ne, tothi, stark_pe (ncell, float32)
//   species per species: llam0 (float64), lower_ev, gpref, grad, gw1, gw2, gstk
//           (float32), unsold (uint8), inv_df, vbar2, lnbase (ncell, float32)
//   shape   nx, ny, nz; slab_nz the planes of each slab
//   geom    ds_cm(3), ds_code(3), pivot_z, ray_offset(2), tol, maser_chi_floor,
//           maser_dtau_max, maser_Inu_max
#include <ATen/ATen.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include <vector>

#include "../../include/m3dgpu.h"

namespace {

void check(int rc, const char *what) {
  if (rc != M3D_OK) {
    char buf[512];
    m3d_last_error(buf, sizeof buf);
    TORCH_CHECK(false, what, ": status ", rc, ": ", buf);
  }
}

// the calling thread's context on the tensor's device, ordered on torch's stream
void on_stream(const at::Tensor &t) {
  TORCH_CHECK(t.is_cuda(), "m3d operators take CUDA tensors");
  const int dev = t.device().index();
  check(m3d_init(dev, 0), "m3d_init");
  cudaStream_t s = at::cuda::getCurrentCUDAStream(dev).stream();
  // torch's default stream is the legacy one (handle 0), which the library names by
  // cudaStreamLegacy; a null handle would select the library's own stream
  check(m3d_set_stream(s ? (void *)s : (void *)0x1), "m3d_set_stream");
}

template <typename T>
T *dptr(const at::Tensor &t, at::ScalarType st, const char *name) {
  TORCH_CHECK(t.is_cuda() && t.is_contiguous(), name, " must be a contiguous CUDA tensor");
  TORCH_CHECK(t.scalar_type() == st, name, " has the wrong dtype");
  return reinterpret_cast<T *>(t.data_ptr());
}

template <typename T>
T *optptr(const c10::optional<at::Tensor> &t, at::ScalarType st, const char *name) {
  return (t.has_value() && t->defined()) ? dptr<T>(*t, st, name) : nullptr;
}

struct Atmos {
  m3d_atmos_t a;
  std::vector<m3d_species_t> sp;
  std::vector<int> slab;
  int64_t ncell;
};

void make_atmos(Atmos &A, at::TensorList cells, at::TensorList species, at::IntArrayRef shape,
                at::IntArrayRef slab_nz, at::ArrayRef<double> geom) {
  TORCH_CHECK(cells.size() == 9, "cells: temp, chi_c, vx, vy, vz, e_kT, ne, tothi, stark_pe");
  TORCH_CHECK(species.size() % 11 == 0, "species: 11 tensors per species");
  TORCH_CHECK(shape.size() == 3, "shape: nx, ny, nz");
  TORCH_CHECK(geom.size() == 13, "geom: ds_cm(3), ds_code(3), pivot_z, ray_offset(2), tol, maser_chi_floor, "
                                 "maser_dtau_max, maser_Inu_max");
  memset(&A.a, 0, sizeof A.a);
  A.a.nx = (int)shape[0];
  A.a.ny = (int)shape[1];
  A.a.nz = (int)shape[2];
  A.ncell = shape[0] * shape[1] * shape[2];
  A.slab.assign(slab_nz.begin(), slab_nz.end());
  if (A.slab.empty()) A.slab.push_back(A.a.nz);
  A.a.nslab = (int)A.slab.size();
  A.a.slab_nz = A.slab.data();
  for (int i = 0; i < 3; i++) { A.a.ds_cm[i] = geom[i]; A.a.ds_code[i] = geom[3 + i]; }
  A.a.pivot_z = geom[6];
  A.a.ray_offset[0] = geom[7];
  A.a.ray_offset[1] = geom[8];
  A.a.tol = geom[9];
  A.a.maser_chi_floor = geom[10];
  A.a.maser_dtau_max = geom[11];
  A.a.maser_Inu_max = geom[12];
  const float **f[9] = {&A.a.temp, &A.a.chi_c, &A.a.vx, &A.a.vy, &A.a.vz, &A.a.e_kT, &A.a.ne, &A.a.tothi,
                        &A.a.stark_pe};
  for (int i = 0; i < 9; i++) {
    TORCH_CHECK(cells[i].numel() == A.ncell, "cell field ", i, " has the wrong size");
    *f[i] = dptr<const float>(cells[i], at::kFloat, "cell field");
  }
  const size_t nsp = species.size() / 11;
  A.sp.assign(nsp, m3d_species_t{});
  for (size_t k = 0; k < nsp; k++) {
    const at::Tensor *s = &species[11 * k];
    m3d_linelist_t &L = A.sp[k].ll;
    memset(&L, 0, sizeof L);
    L.nline = (int)s[0].numel();
    L.llam0 = dptr<const double>(s[0], at::kDouble, "llam0");
    L.lower_ev = dptr<const float>(s[1], at::kFloat, "lower_ev");
    L.gpref = dptr<const float>(s[2], at::kFloat, "gpref");
    L.grad = dptr<const float>(s[3], at::kFloat, "grad");
    L.gw1 = dptr<const float>(s[4], at::kFloat, "gw1");
    L.gw2 = dptr<const float>(s[5], at::kFloat, "gw2");
    L.gstk = dptr<const float>(s[6], at::kFloat, "gstk");
    L.unsold = dptr<const unsigned char>(s[7], at::kByte, "unsold");
    for (int i = 1; i < 8; i++) TORCH_CHECK(s[i].numel() == L.nline, "line array ", i, " has the wrong size");
    A.sp[k].inv_df = dptr<const float>(s[8], at::kFloat, "inv_df");
    A.sp[k].vbar2 = dptr<const float>(s[9], at::kFloat, "vbar2");
    A.sp[k].lnbase = dptr<const float>(s[10], at::kFloat, "lnbase");
    for (int i = 8; i < 11; i++) TORCH_CHECK(s[i].numel() == A.ncell, "species field has the wrong size");
  }
  A.a.nspecies = (int)nsp;
  A.a.species = A.sp.data();
}

std::tuple<at::Tensor, at::Tensor, at::Tensor> lte_synthesis(at::TensorList cells, at::TensorList species,
                                                             at::IntArrayRef shape, at::IntArrayRef slab_nz,
                                                             at::ArrayRef<double> geom, const at::Tensor &nu,
                                                             const at::Tensor &llam, at::ArrayRef<double> vec,
                                                             at::ArrayRef<double> wmu, bool fp64, bool return_itop) {
  on_stream(nu);
  Atmos A;
  make_atmos(A, cells, species, shape, slab_nz, geom);
  const int nf = (int)nu.numel(), nray = (int)wmu.size();
  TORCH_CHECK((int)vec.size() == 3 * nray, "vec: 3 per ray");
  auto fo = nu.options().dtype(at::kFloat);
  at::Tensor ie = at::empty({nray, nf}, fo), flux = at::empty({nf}, fo), itop;
  if (return_itop) itop = at::empty({nray, shape[1], shape[0], nf}, nu.options().dtype(fp64 ? at::kDouble : at::kFloat));
  check(m3d_lte_synthesis(&A.a, nf, dptr<const double>(nu, at::kDouble, "nu"),
                          dptr<const double>(llam, at::kDouble, "llam"), nray, vec.data(), wmu.data(),
                          return_itop ? itop.data_ptr() : nullptr, ie.data_ptr<float>(), flux.data_ptr<float>(),
                          M3D_DEVICE_PTRS | (fp64 ? M3D_FP64 : 0u)),
        "m3d_lte_synthesis");
  return {ie, flux, itop};
}

std::tuple<at::Tensor, at::Tensor> lte_transfer_units(at::TensorList cells, at::TensorList species,
                                                      at::IntArrayRef shape, at::ArrayRef<double> geom,
                                                      const at::Tensor &nu, const at::Tensor &llam,
                                                      at::ArrayRef<double> vec, bool fp64) {
  on_stream(nu);
  Atmos A;
  make_atmos(A, cells, species, shape, {}, geom);
  TORCH_CHECK(vec.size() == 3, "vec: one direction");
  const int nf = (int)nu.numel();
  auto o = nu.options().dtype(fp64 ? at::kDouble : at::kFloat);
  at::Tensor chi = at::empty({A.ncell, nf}, o), S = at::empty({A.ncell, nf}, o);
  check(m3d_lte_transfer_units(&A.a, nf, dptr<const double>(nu, at::kDouble, "nu"),
                               dptr<const double>(llam, at::kDouble, "llam"), vec.data(), chi.data_ptr(), S.data_ptr(),
                               M3D_DEVICE_PTRS | (fp64 ? M3D_FP64 : 0u)),
        "m3d_lte_transfer_units");
  return {chi, S};
}

std::vector<at::Tensor> lte_synthesis_adjoint(at::TensorList cells, at::TensorList species, at::IntArrayRef shape,
                                              at::IntArrayRef slab_nz, at::ArrayRef<double> geom,
                                              const at::Tensor &nu, const at::Tensor &llam, at::ArrayRef<double> vec,
                                              at::ArrayRef<double> wmu, const at::Tensor &g_flux) {
  on_stream(nu);
  Atmos A;
  make_atmos(A, cells, species, shape, slab_nz, geom);
  const int nf = (int)nu.numel(), nray = (int)wmu.size();
  TORCH_CHECK((int)vec.size() == 3 * nray, "vec: 3 per ray");
  int64_t nline = 0;
  for (auto &s : A.sp) nline += s.ll.nline;
  auto fo = nu.options().dtype(at::kFloat);
  const int64_t nsp = std::max<int64_t>((int64_t)A.sp.size(), 1);
  std::vector<at::Tensor> g = {at::zeros({A.ncell}, fo), at::zeros({A.ncell}, fo), at::zeros({A.ncell}, fo),
                               at::zeros({nsp, A.ncell}, fo), at::zeros({nsp, A.ncell}, fo),
                               at::zeros({std::max<int64_t>(nline, 1)}, fo)};
  m3d_lte_grad_t gr = {g[0].data_ptr<float>(), g[1].data_ptr<float>(), g[2].data_ptr<float>(),
                       g[3].data_ptr<float>(), g[4].data_ptr<float>(), g[5].data_ptr<float>()};
  check(m3d_lte_synthesis_adjoint(&A.a, nf, dptr<const double>(nu, at::kDouble, "nu"),
                                  dptr<const double>(llam, at::kDouble, "llam"), nray, vec.data(), wmu.data(),
                                  dptr<const float>(g_flux, at::kFloat, "g_flux"), &gr, M3D_DEVICE_PTRS),
        "m3d_lte_synthesis_adjoint");
  return g;
}

m3d_slab_t make_slab(at::IntArrayRef dims, int64_t dir, at::ArrayRef<double> ds, at::ArrayRef<double> vec,
                     bool get_psi, bool split_rates, double maser_dtau_max, double maser_Inu_max) {
  TORCH_CHECK(dims.size() == 4 && ds.size() == 3 && vec.size() == 3, "dims (nf, nx, ny, nz), ds(3), vec(3)");
  m3d_slab_t s;
  memset(&s, 0, sizeof s);
  s.nf = (int)dims[0]; s.nx = (int)dims[1]; s.ny = (int)dims[2]; s.nz = (int)dims[3];
  s.dir = (int)dir;
  s.get_psi = get_psi;
  s.split_rates = split_rates;
  for (int i = 0; i < 3; i++) { s.ds[i] = ds[i]; s.vec[i] = vec[i]; }
  s.maser_dtau_max = maser_dtau_max;
  s.maser_Inu_max = maser_Inu_max;
  return s;
}

void formal_solve(int64_t solver, const at::Tensor &work, const c10::optional<at::Tensor> &psi,
                  const c10::optional<at::Tensor> &irem, const c10::optional<at::Tensor> &escape,
                  const c10::optional<at::Tensor> &chi500, const c10::optional<at::Tensor> &chi500_up,
                  const c10::optional<at::Tensor> &g500, const c10::optional<at::Tensor> &eta_row,
                  const c10::optional<at::Tensor> &eta_mask, at::IntArrayRef dims, int64_t dir,
                  at::ArrayRef<double> ds, at::ArrayRef<double> vec, bool get_psi, bool split_rates,
                  double maser_dtau_max, double maser_Inu_max, c10::optional<at::ArrayRef<double>> rotate) {
  on_stream(work);
  const bool f64 = work.scalar_type() == at::kDouble;
  const auto st = f64 ? at::kDouble : at::kFloat;
  m3d_slab_t s = make_slab(dims, dir, ds, vec, get_psi, split_rates, maser_dtau_max, maser_Inu_max);
  unsigned flags = M3D_DEVICE_PTRS | (f64 ? M3D_FP64 : 0u);
  const double *rds = nullptr, *roff = nullptr;
  double rb2p = 0.0;
  if (rotate.has_value()) {
    TORCH_CHECK(rotate->size() == 6, "rotate: ds_code(3), bot2pivot, ray_offset(2)");
    rds = rotate->data();
    rb2p = (*rotate)[3];
    roff = rotate->data() + 4;
    flags |= M3D_ROTATE;
  }
  check(m3d_formal_solve((int)solver, &s, dptr<void>(work, st, "work"), optptr<void>(psi, st, "psi"),
                         optptr<void>(irem, st, "irem"), optptr<void>(escape, st, "escape"),
                         optptr<const float>(chi500, at::kFloat, "chi500"),
                         optptr<const float>(chi500_up, at::kFloat, "chi500_up"),
                         optptr<const float>(g500, at::kFloat, "g500"), optptr<const int>(eta_row, at::kInt, "eta_row"),
                         optptr<const unsigned char>(eta_mask, at::kByte, "eta_mask"), rds, rb2p, roff, flags),
        "m3d_formal_solve");
}

void rotate_array(const at::Tensor &work, at::IntArrayRef dims, at::ArrayRef<double> vec,
                  at::ArrayRef<double> ds_code, double bot2pivot, at::ArrayRef<double> ray_offset) {
  on_stream(work);
  const bool f64 = work.scalar_type() == at::kDouble;
  TORCH_CHECK(ds_code.size() == 3 && ray_offset.size() == 2, "ds_code(3), ray_offset(2)");
  m3d_slab_t s = make_slab(dims, 1, {1.0, 1.0, 1.0}, vec, false, false, 2.0, 1e30);
  check(m3d_rotate_array(&s, dptr<void>(work, f64 ? at::kDouble : at::kFloat, "work"), ds_code.data(), bot2pivot,
                         ray_offset.data(), M3D_DEVICE_PTRS | (f64 ? M3D_FP64 : 0u)),
        "m3d_rotate_array");
}

void line_opacity(at::TensorList linelist, const at::Tensor &llam, const at::Tensor &chi, const at::Tensor &eta,
                  const at::Tensor &cont, const at::Tensor &logref, at::TensorList cellf, double tol,
                  double line_reject_frac) {
  on_stream(chi);
  TORCH_CHECK(linelist.size() == 8, "linelist: llam0, lower_ev, gpref, grad, gw1, gw2, gstk, unsold");
  TORCH_CHECK(cellf.size() == 8, "cells: vproj, inv_df, vbar2, e_kT, lnbase, ne, tothi, stark_pe");
  m3d_linelist_t L;
  memset(&L, 0, sizeof L);
  L.nline = (int)linelist[0].numel();
  L.llam0 = dptr<const double>(linelist[0], at::kDouble, "llam0");
  L.lower_ev = dptr<const float>(linelist[1], at::kFloat, "lower_ev");
  L.gpref = dptr<const float>(linelist[2], at::kFloat, "gpref");
  L.grad = dptr<const float>(linelist[3], at::kFloat, "grad");
  L.gw1 = dptr<const float>(linelist[4], at::kFloat, "gw1");
  L.gw2 = dptr<const float>(linelist[5], at::kFloat, "gw2");
  L.gstk = dptr<const float>(linelist[6], at::kFloat, "gstk");
  L.unsold = dptr<const unsigned char>(linelist[7], at::kByte, "unsold");
  const int nf = (int)llam.numel(), ncell = (int)cellf[0].numel();
  const float *c[8];
  for (int i = 0; i < 8; i++) c[i] = dptr<const float>(cellf[i], at::kFloat, "cell field");
  check(m3d_line_opacity(&L, nf, dptr<const double>(llam, at::kDouble, "llam"), ncell,
                         dptr<float>(chi, at::kFloat, "chi"), dptr<float>(eta, at::kFloat, "eta"),
                         dptr<const float>(cont, at::kFloat, "cont"), dptr<const float>(logref, at::kFloat, "logref"),
                         c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], nullptr, 0, 0, (float)tol,
                         (float)line_reject_frac, nullptr, nullptr, nullptr, M3D_DEVICE_PTRS),
        "m3d_line_opacity");
}

void integrate_intensity(double wmu, const at::Tensor &inu, const at::Tensor &psi, const at::Tensor &Jnu,
                         const at::Tensor &PsiJ) {
  on_stream(inu);
  check(m3d_integrate_intensity((int)inu.numel(), (float)wmu, dptr<const float>(inu, at::kFloat, "inu"),
                                dptr<const float>(psi, at::kFloat, "psi"), dptr<float>(Jnu, at::kFloat, "Jnu"),
                                dptr<float>(PsiJ, at::kFloat, "PsiJ"), M3D_DEVICE_PTRS),
        "m3d_integrate_intensity");
}

at::Tensor qlg_bot_profile(const at::Tensor &a, const at::Tensor &q, const at::Tensor &vpr, const at::Tensor &idf) {
  on_stream(a);
  at::Tensor h = at::empty_like(q);
  check(m3d_qlg_bot_profile((int)a.numel(), dptr<const float>(a, at::kFloat, "a"), dptr<const float>(q, at::kFloat, "q"),
                            dptr<const float>(vpr, at::kFloat, "vpr"), dptr<const float>(idf, at::kFloat, "idf"),
                            h.data_ptr<float>(), M3D_DEVICE_PTRS),
        "m3d_qlg_bot_profile");
  return h;
}

// update_populations of every cell.  atom and cells are the addresses of the host
// descriptors m3d_atom_t and m3d_col_cells_t (their arrays device memory), as the
// library's Python front end builds them; params: max_update, sor_w, min_pop_frac,
// conv_pop_floor, tmax_update, cswitch.  Returns maxerr, epos_cell, epos_level,
// nclamp, ntot, nonfinite_cell (float64 on the host).
at::Tensor stateq_update(int64_t atom, int64_t cells, int64_t solver, at::ArrayRef<double> params, const at::Tensor &b,
                         const at::Tensor &nstar, const at::Tensor &totn, const at::Tensor &e_kT,
                         const at::Tensor &gamma_ij, const at::Tensor &gamma_ji, const c10::optional<at::Tensor> &cup,
                         const at::Tensor &lvlerr) {
  on_stream(b);
  TORCH_CHECK(params.size() == 6, "params: max_update, sor_w, min_pop_frac, conv_pop_floor, tmax_update, cswitch");
  m3d_se_params_t p = {params[0], params[1], params[2], params[3], params[4], params[5], (int)solver, 0};
  m3d_se_result_t r;
  memset(&r, 0, sizeof r);
  TORCH_CHECK(!lvlerr.is_cuda() && lvlerr.scalar_type() == at::kDouble, "lvlerr: a float64 host tensor");
  const int rc = m3d_stateq_update(reinterpret_cast<const m3d_atom_t *>(atom), &p, (int)totn.size(-1),
                                   dptr<double>(b, at::kDouble, "b"), dptr<const double>(nstar, at::kDouble, "nstar"),
                                   dptr<const double>(totn, at::kDouble, "totn"),
                                   dptr<const double>(e_kT, at::kDouble, "e_kT"),
                                   reinterpret_cast<const m3d_col_cells_t *>(cells),
                                   dptr<const float>(gamma_ij, at::kFloat, "gamma_ij"),
                                   dptr<const float>(gamma_ji, at::kFloat, "gamma_ji"),
                                   optptr<const double>(cup, at::kDouble, "cup"), lvlerr.data_ptr<double>(), &r,
                                   M3D_DEVICE_PTRS);
  if (rc != M3D_ENONFINITE) check(rc, "m3d_stateq_update");
  at::Tensor out = at::empty({7}, at::TensorOptions().dtype(at::kDouble));
  double *o = out.data_ptr<double>();
  o[0] = r.maxerr; o[1] = (double)r.epos_cell; o[2] = r.epos_level; o[3] = (double)r.nclamp; o[4] = (double)r.ntot;
  o[5] = (double)r.nonfinite_cell; o[6] = rc;
  return out;
}

}  // namespace

TORCH_LIBRARY(m3d, m) {
  m.def("lte_synthesis(Tensor[] cells, Tensor[] species, int[] shape, int[] slab_nz, float[] geom, Tensor nu, "
        "Tensor llam, float[] vec, float[] wmu, bool fp64, bool return_itop) -> (Tensor, Tensor, Tensor)");
  m.def("lte_transfer_units(Tensor[] cells, Tensor[] species, int[] shape, float[] geom, Tensor nu, Tensor llam, "
        "float[] vec, bool fp64) -> (Tensor, Tensor)");
  m.def("lte_synthesis_adjoint(Tensor[] cells, Tensor[] species, int[] shape, int[] slab_nz, float[] geom, "
        "Tensor nu, Tensor llam, float[] vec, float[] wmu, Tensor g_flux) -> Tensor[]");
  m.def("formal_solve(int solver, Tensor(a!) work, Tensor(b!)? psi, Tensor(c!)? irem, Tensor(d!)? escape, "
        "Tensor? chi500, Tensor? chi500_up, Tensor? g500, Tensor? eta_row, Tensor? eta_mask, int[] dims, int dir, "
        "float[] ds, float[] vec, bool get_psi, bool split_rates, float maser_dtau_max, float maser_Inu_max, "
        "float[]? rotate) -> ()");
  m.def("rotate_array(Tensor(a!) work, int[] dims, float[] vec, float[] ds_code, float bot2pivot, "
        "float[] ray_offset) -> ()");
  m.def("line_opacity(Tensor[] linelist, Tensor llam, Tensor(a!) chi, Tensor(b!) eta, Tensor cont, Tensor logref, "
        "Tensor[] cells, float tol, float line_reject_frac) -> ()");
  m.def("integrate_intensity(float wmu, Tensor inu, Tensor psi, Tensor(a!) Jnu, Tensor(b!) PsiJ) -> ()");
  m.def("qlg_bot_profile(Tensor a, Tensor q, Tensor vpr, Tensor idf) -> Tensor");
  m.def("stateq_update(int atom, int cells, int solver, float[] params, Tensor(a!) b, Tensor nstar, Tensor totn, "
        "Tensor e_kT, Tensor gamma_ij, Tensor gamma_ji, Tensor? cup, Tensor(b!) lvlerr) -> Tensor");
}

TORCH_LIBRARY_IMPL(m3d, CUDA, m) {
  m.impl("lte_synthesis", &lte_synthesis);
  m.impl("lte_transfer_units", &lte_transfer_units);
  m.impl("lte_synthesis_adjoint", &lte_synthesis_adjoint);
  m.impl("formal_solve", &formal_solve);
  m.impl("rotate_array", &rotate_array);
  m.impl("line_opacity", &line_opacity);
  m.impl("integrate_intensity", &integrate_intensity);
  m.impl("qlg_bot_profile", &qlg_bot_profile);
  m.impl("stateq_update", &stateq_update);
}

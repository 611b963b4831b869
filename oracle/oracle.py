"""ctypes front end of the CPU oracle (oracle/m3d_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it as the checker.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libm3d_oracle.so")

F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

LINEAR, LINEAR2, QUADRATIC, SHORT_LINEAR, SHORT_LINEAR2 = range(5)
BND_NONE, BND_ZERO, BND_PCHIP, BND_LTE = range(4)


class Slab(C.Structure):
    """or_slab_t: one depth slab of one direction (rt_patch_t's sweep state)."""

    _fields_ = [("nf", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dir", C.c_int), ("get_psi", C.c_int), ("split_rates", C.c_int), ("pad", C.c_int),
                ("ds", C.c_double * 3), ("vec", C.c_double * 3),
                ("maser_dtau_max", C.c_double), ("maser_Inu_max", C.c_double)]


class LineList(C.Structure):
    _fields_ = [("nline", C.c_int), ("llam0", C.c_void_p), ("lower_ev", C.c_void_p),
                ("gpref", C.c_void_p), ("grad", C.c_void_p), ("gw1", C.c_void_p),
                ("gw2", C.c_void_p), ("gstk", C.c_void_p), ("unsold", C.c_void_p),
                ("lev_i", C.c_void_p), ("lev_j", C.c_void_p), ("active", C.c_void_p),
                ("reach_in", C.c_void_p)]


def build() -> str:
    """Compile the oracle with its Makefile (gcc only); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def make_slab(nf, nx, ny, nz, dir, ds, vec, get_psi=False, split_rates=False,
              maser_dtau_max=2.0, maser_Inu_max=1e30) -> Slab:
    s = Slab()
    s.nf, s.nx, s.ny, s.nz, s.dir = nf, nx, ny, nz, dir
    s.get_psi, s.split_rates = int(get_psi), int(split_rates)
    s.ds[:] = [float(v) for v in ds]
    s.vec[:] = [float(v) for v in vec]
    s.maser_dtau_max, s.maser_Inu_max = maser_dtau_max, maser_Inu_max
    return s


# ---- K0 ------------------------------------------------------------------------
def _vec1(fn, x, dtype, nout):
    x = np.ascontiguousarray(x, dtype)
    outs = [np.empty_like(x) for _ in range(nout)]
    getattr(lib(), fn)(C.c_int(x.size), _p(x), *[_p(o) for o in outs])
    return outs if nout > 1 else outs[0]


def exp_neg(t):
    return _vec1("or_exp_neg_f32", t, np.float32, 2)


def exp_neg0(t):
    return _vec1("or_exp_neg0_f32", t, np.float32, 2)


def exp4(x):
    return _vec1("or_exp4_f32", x, np.float32, 1)


def logf(x):
    return _vec1("or_log_f32", x, np.float32, 1)


def linear_weights(t, fp64=False):
    return _vec1("or_linear_weights_f64" if fp64 else "or_linear_weights_f32", t,
                 np.float64 if fp64 else np.float32, 4)


def parab_moments(t, fp64=False):
    return _vec1("or_parab_moments_f64" if fp64 else "or_parab_moments_f32", t,
                 np.float64 if fp64 else np.float32, 4)


def bezier3_weights(t):
    """(w0, w1, w2, w3) of bezier3_weights (rt_solvers_mod.f90:1280-1331), fp32."""
    return _vec1("or_bezier3_weights_f32", t, np.float32, 4)


def set_stencil(ds, vec):
    ds = (C.c_double * 3)(*ds)
    vec = (C.c_double * 3)(*vec)
    xk, yk = (C.c_double * 4)(), (C.c_double * 4)()
    u1, u2, dsup = C.c_int(), C.c_int(), C.c_double()
    lib().or_set_stencil(ds, vec, xk, yk, C.byref(u1), C.byref(u2), C.byref(dsup))
    return np.array(xk[:]), np.array(yk[:]), u1.value, u2.value, dsup.value


# ---- QLG -------------------------------------------------------------------------
_tables = None


def qlg_tables():
    global _tables
    if _tables is None:
        tgx = np.empty(9020, np.float32)
        th2x = np.empty(9020, np.float32)
        lib().or_qlg_tables(_p(tgx), _p(th2x))
        _tables = (tgx, th2x)
    return _tables


_tables64 = None


def qlg_tables_f64():
    """qlg_init's two tables in fp64 (the plain FP64 path's tables)."""
    global _tables64
    if _tables64 is None:
        tgx = np.empty(9020, np.float64)
        th2x = np.empty(9020, np.float64)
        lib().or_qlg_tables_f64(_p(tgx), _p(th2x))
        _tables64 = (tgx, th2x)
    return _tables64


def opacity_f64(ll: dict, llam, chl, xhat, vproj, cells: dict, tol=1e-4):
    """The plain FP64 line opacity of one species, accumulated in place on chl
    (ncell, nf) f64.  xhat (ncell, nf) and vproj (ncell,) f64; cells: inv_df, vbar2,
    e_kT, lnbase, ne, tothi, stark_pe (ncell,) f32.  tol is the float tolerance."""
    tgx, th2x = qlg_tables_f64()
    s, keep = make_linelist(ll)
    llam = np.ascontiguousarray(llam, np.float64)
    assert chl.dtype == np.float64 and chl.flags.c_contiguous
    xh = np.ascontiguousarray(xhat, np.float64)
    vp = np.ascontiguousarray(vproj, np.float64)
    cf = {k: np.ascontiguousarray(cells[k], np.float32) for k in
          ("inv_df", "vbar2", "e_kT", "lnbase", "ne", "tothi", "stark_pe")}
    f = lib().or_opacity_f64
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_void_p] + [C.c_void_p] * 7 + [C.c_double]
    rc = f(_p(tgx), _p(th2x), C.byref(s), llam.size, _p(llam), vp.size, _p(chl), _p(xh), _p(vp),
           *[_p(cf[k]) for k in ("inv_df", "vbar2", "e_kT", "lnbase", "ne", "tothi", "stark_pe")],
           float(np.float32(tol)))
    assert rc == 0
    del keep


def qlg_ref_f64(a, v):
    v = np.ascontiguousarray(v, np.float64)
    out = np.empty_like(v)
    f = lib().or_qlg_ref_f64
    f.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p]
    for i, vi in enumerate(v):
        tmp = np.empty(1)
        f(float(a), float(vi), 0.0, 1, _p(tmp))
        out[i] = tmp[0]
    return out


def qlg_bot_sweep(a, v0, dv, n):
    tgx, th2x = qlg_tables()
    K = np.empty(n, np.float32)
    f = lib().or_qlg_bot_sweep
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]
    f(_p(tgx), _p(th2x), a, v0, dv, n, _p(K))
    return K


def qlg_bot_profile(a, q, vpr, idf):
    tgx, th2x = qlg_tables()
    a, q, vpr, idf = (np.ascontiguousarray(x, np.float32) for x in (a, q, vpr, idf))
    h = np.empty_like(a)
    lib().or_qlg_bot_profile(_p(tgx), _p(th2x), C.c_int(a.size), _p(a), _p(q), _p(vpr), _p(idf), _p(h))
    return h


def qlg_bot_line_sweep(D, gL, S, ref, lnq, llam, llc, pos, idl, cap=np.finfo(np.float32).max):
    tgx, th2x = qlg_tables()
    llam = np.ascontiguousarray(llam, np.float64)
    K = np.zeros(llam.size, np.float32)
    fa, fb, hw = C.c_int(), C.c_int(), C.c_float()
    f = lib().or_qlg_bot_line_sweep
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                  C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_float,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    n = f(_p(tgx), _p(th2x), D, gL, S, ref, lnq, llam.size, _p(llam), llc, pos, idl, cap,
          C.byref(fa), C.byref(fb), C.byref(hw), _p(K))
    return fa.value, fb.value, hw.value, K[:n]


# ---- line opacity -----------------------------------------------------------------------
def make_linelist(ll: dict) -> tuple[LineList, list]:
    """ll: dict of numpy arrays (llam0 f64; lower_ev, gpref, grad, gw1, gw2, gstk f32;
    unsold u8; optional lev_i, lev_j i32, active u8).  Returns the struct and the
    arrays it points into (keep them alive)."""
    keep = []

    def arr(name, dt):
        if name not in ll or ll[name] is None:
            return None
        a = np.ascontiguousarray(ll[name], dt)
        keep.append(a)
        return _p(a)

    s = LineList()
    s.nline = int(len(ll["llam0"]))
    s.llam0 = arr("llam0", np.float64)
    for k in ("lower_ev", "gpref", "grad", "gw1", "gw2", "gstk"):
        setattr(s, k, arr(k, np.float32))
    s.unsold = arr("unsold", np.uint8)
    s.lev_i = arr("lev_i", np.int32)
    s.lev_j = arr("lev_j", np.int32)
    s.active = arr("active", np.uint8)
    s.reach_in = arr("reach_in", np.float32)
    return s, keep


def select_lines(ll: dict, llam, vmax: float):
    """select_lines: the selected 0-based line indices."""
    s, keep = make_linelist(ll)
    llam = np.ascontiguousarray(llam, np.float64)
    sel = np.zeros(max(s.nline, 1), np.int32)
    n = lib().or_select_lines(C.byref(s), C.c_int(llam.size), _p(llam), C.c_float(vmax), _p(sel))
    return sel[:n]


def add_opacity_equi(ll: dict, llam, chi, eta, cont, logref, cells: dict, dep_mem=None,
                     nlevel=0, do_nlte=False, tol=1e-4, line_reject_frac=0.0, one_m_eps=None, chi_scat=None):
    """In place on chi/eta (nf, ncell) f32.  cells: vproj, inv_df, vbar2, e_kT, lnbase,
    ne, tothi, stark_pe (ncell,) f32.  one_m_eps, chi_scat: the line_scattering split
    (chi_scat accumulated in place).  Returns (used, strength, reach)."""
    tgx, th2x = qlg_tables()
    s, keep = make_linelist(ll)
    nl = s.nline
    used = np.zeros(nl, np.uint8)
    strength = np.zeros(nl, np.float32)
    reach = np.zeros(nl, np.float32)
    llam = np.ascontiguousarray(llam, np.float64)
    ncell = chi.shape[0] if chi.ndim == 2 and chi.shape[1] == llam.size else chi.size // llam.size
    cf = {k: np.ascontiguousarray(cells[k], np.float32) for k in
          ("vproj", "inv_df", "vbar2", "e_kT", "lnbase", "ne", "tothi", "stark_pe")}
    dm = None if dep_mem is None else np.ascontiguousarray(dep_mem, np.float32)
    for a in (chi, eta):
        assert a.dtype == np.float32 and a.flags.c_contiguous
    om = None if one_m_eps is None else np.ascontiguousarray(one_m_eps, np.float32)
    if chi_scat is not None:
        assert chi_scat.dtype == np.float32 and chi_scat.flags.c_contiguous and om is not None
    rc = lib().or_add_opacity_equi_scat(
        _p(tgx), _p(th2x), C.byref(s), C.c_int(llam.size), _p(llam), C.c_int(ncell),
        _p(chi), _p(eta), _p(np.ascontiguousarray(cont, np.float32)),
        _p(np.ascontiguousarray(logref, np.float32)),
        *[_p(cf[k]) for k in ("vproj", "inv_df", "vbar2", "e_kT", "lnbase", "ne", "tothi", "stark_pe")],
        _p(dm), C.c_int(nlevel), C.c_int(int(do_nlte)), C.c_float(tol), C.c_float(line_reject_frac),
        _p(used), _p(strength), _p(reach), _p(om), _p(chi_scat))
    assert rc == 0
    del keep
    return used, strength, reach


# ---- background / units ------------------------------------------------------------------
def lte_background(nu, temp):
    nu = np.ascontiguousarray(nu, np.float64)
    temp = np.ascontiguousarray(temp, np.float32)
    beta = np.empty((temp.size, nu.size), np.float32)
    Bnu = np.empty_like(beta)
    lib().or_lte_background(C.c_int(nu.size), C.c_int(temp.size), _p(nu), _p(temp), _p(beta), _p(Bnu))
    return beta, Bnu


def lte_work(chi_c, beta, Bnu):
    chi_c = np.ascontiguousarray(chi_c, np.float32)
    xhat = np.empty_like(beta)
    ehat = np.empty_like(beta)
    nc, nf = beta.shape
    lib().or_lte_work(C.c_int(nf), C.c_int(nc), _p(chi_c), _p(beta), _p(Bnu), _p(xhat), _p(ehat))
    return xhat, ehat


def logref(xhat, tol=1e-4):
    xhat = np.ascontiguousarray(xhat, np.float32)
    out = np.empty_like(xhat)
    f = lib().or_logref
    f.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_void_p]
    f(xhat.size, _p(xhat), tol, _p(out))
    return out


def work_to_transfer_units(w1, w2, beta, maser_chi_floor=1e-4, suppress_masers=False):
    nc, nf = beta.shape
    f = lib().or_work_to_transfer_units
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int]
    return f(nf, nc, _p(w1), _p(w2), _p(beta), maser_chi_floor, int(suppress_masers))


# ---- solvers -----------------------------------------------------------------------------
def formal_solve(solver, slab: Slab, work, psi=None, irem=None, escape=None, chi500=None,
                 chi500_up=None, g500=None, eta_row=None, eta_mask=None):
    fp64 = work.dtype == np.float64
    fn = lib().or_formal_solve_f64 if fp64 else lib().or_formal_solve_f32
    rc = fn(C.c_int(solver), C.byref(slab), _p(work), _p(psi), _p(irem), _p(escape),
            _p(chi500), _p(chi500_up), _p(g500), _p(eta_row), _p(eta_mask))
    if rc:
        raise RuntimeError(f"oracle formal_solve rc={rc}")


def long_char_hermite(slab: Slab, work, psi, beta, pe, dpe_dz, dlnt_dz, temp, hknu, ghost=None,
                      code_length=1.0):
    """long_char_hermite (rt_solvers_mod.f90:1052-1504) in place on work (fp32).
    ghost: dict pe, dpe_dz, dlnt_dz, temp (ny, nx) of the upstream ghost, or None
    for the zeroed top ghost."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    g = ghost or {}
    args = [f32(x) for x in (beta, pe, dpe_dz, dlnt_dz, temp, hknu)]
    gargs = [None if not g else f32(g[k]) for k in ("pe", "dpe_dz", "dlnt_dz", "temp")]
    assert work.dtype == np.float32 and work.flags.c_contiguous
    rc = lib().or_long_char_hermite(C.byref(slab), _p(work), _p(psi), *[_p(a) for a in args],
                                    *[_p(a) for a in gargs], C.c_double(code_length))
    if rc:
        raise RuntimeError(f"oracle long_char_hermite rc={rc}")


def long_char_hermite2(slab: Slab, work, psi, pe, dpe_dz, ghost=None, ghost_kind=0, code_length=1.0):
    """long_char_hermite2 (rt_solvers_mod.f90:1536-1895) in place on work (fp32).
    ghost: dict pe, dpe_dz (ny, nx) of the upstream ghost, or None for the zeroed
    top ghost; ghost_kind 1 = an upstream neighbour's exit plane, 2 = the bottom's
    ghost model (they differ only for nz == 2)."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    g = [None, None] if not ghost else [f32(ghost["pe"]), f32(ghost["dpe_dz"])]
    kind = 0 if not ghost else (ghost_kind or 2)
    pe, dpe_dz = f32(pe), f32(dpe_dz)
    assert work.dtype == np.float32 and work.flags.c_contiguous
    rc = lib().or_long_char_hermite2(C.byref(slab), _p(work), _p(psi), _p(pe), _p(dpe_dz), _p(g[0]), _p(g[1]),
                                     C.c_int(kind), C.c_double(code_length))
    if rc:
        raise RuntimeError(f"oracle long_char_hermite2 rc={rc}")


def short_char_hermite(slab: Slab, work, psi, irem, esc, beta, pe, dpe_dx, dpe_dy, dpe_dz, dlnt_dx, dlnt_dy,
                       dlnt_dz, temp, hknu, code_length=1.0):
    """short_char_hermite (rt_solvers_mod.f90:1917-2248) in place on work (fp32);
    psi, irem, esc (nz, ny, nx, nf) or None as get_psi / split_rates ask."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    args = [f32(a) for a in (beta, pe, dpe_dx, dpe_dy, dpe_dz, dlnt_dx, dlnt_dy, dlnt_dz, temp, hknu)]
    assert work.dtype == np.float32 and work.flags.c_contiguous
    rc = lib().or_short_char_hermite(C.byref(slab), _p(work), _p(psi), _p(irem), _p(esc), *[_p(a) for a in args],
                                     C.c_double(code_length))
    if rc:
        raise RuntimeError(f"oracle short_char_hermite rc={rc}")


def rotate_array(slab: Slab, work, ds_code, bot2pivot, ray_offset=(0.0, 0.0)):
    fp64 = work.dtype == np.float64
    fn = lib().or_rotate_array_f64 if fp64 else lib().or_rotate_array_f32
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
    fn(C.byref(slab), _p(work), (C.c_double * 3)(*ds_code), float(bot2pivot), (C.c_double * 2)(*ray_offset))


def upstream_boundary(slab: Slab, work, mode, mem=None, ds3_code=1.0, ghost_r500=None,
                      ghost_temp=None, nu=None):
    fp64 = work.dtype == np.float64
    fn = lib().or_upstream_boundary_f64 if fp64 else lib().or_upstream_boundary_f32
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_float, C.c_void_p,
                   C.c_void_p, C.c_void_p]
    fn(C.byref(slab), _p(work), mode, _p(mem), ds3_code, _p(ghost_r500), _p(ghost_temp), _p(nu))


def save_intensity(nu, I_top, wmu):
    """I_top (nmu, ny, nx, nf) f32 -> (ie (nmu, nf), flux (nf,))."""
    nu = np.ascontiguousarray(nu, np.float64)
    I_top = np.ascontiguousarray(I_top, np.float32)
    wmu = np.ascontiguousarray(wmu, np.float64)
    nmu, ny, nx, nf = I_top.shape
    ie = np.empty((nmu, nf), np.float32)
    flux = np.empty(nf, np.float32)
    lib().or_save_intensity(C.c_int(nf), C.c_int(nx), C.c_int(ny), C.c_int(nmu), _p(nu), _p(I_top),
                            _p(wmu), _p(ie), _p(flux))
    return ie, flux


def integrate_intensity(wmu, work3, psi, Jnu, PsiJ):
    f = lib().or_integrate_intensity
    f.argtypes = [C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f(work3.size, 1, wmu, _p(work3), _p(psi), _p(Jnu), _p(PsiJ))

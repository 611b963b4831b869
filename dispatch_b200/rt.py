"""Array-level wrappers of the libm3dgpu.so entry points.

numpy arguments are host buffers; torch CUDA tensors are passed as device
pointers (M3D_DEVICE_PTRS).  All arrays keep the reference's Fortran layout,
frequency fastest; in numpy C order that is the reversed shape, e.g. work is
(3, nz+2, ny, nx, nf).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (DEVICE_PTRS, FP64, LINE_DIAG, ROTATE, Atmos, LineList, Species, check, init, lib, order_after_torch,
               ptr)

_F32 = np.float32


def _is_dev(*arrays) -> bool:
    for a in arrays:
        if a is not None and not isinstance(a, np.ndarray):
            order_after_torch(a)
            return True
    return False


def _flags(arrays, extra=0) -> int:
    f = extra
    if _is_dev(*arrays):
        f |= DEVICE_PTRS
    for a in arrays:
        if a is None:
            continue
        if str(getattr(a, "dtype", "")) in ("float64", "torch.float64"):
            f |= FP64
            break
    return f


def weights(which: int, t, fp64: bool = False):
    """K0 elementwise: 0 exp_neg (E, u0), 1 linear_weights (E, W, Psi, Esc),
    2 parab_moments (E, U0, U1, q), 3 exp4, 4 the library's fp32 log,
    5 bezier3_weights (w0, w1, w2, w3)."""
    init()
    dt = np.float64 if fp64 else np.float32
    t = np.ascontiguousarray(t, dt)
    nout = 2 if which == 0 else (1 if which in (3, 4) else 4)
    outs = [np.empty_like(t) for _ in range(nout)] + [None] * (4 - nout)
    check(lib().m3d_weights(C.c_int(which), C.c_int(t.size), ptr(t), *[ptr(o) for o in outs],
                            C.c_uint(FP64 if fp64 else 0)), "m3d_weights")
    return outs[:nout] if nout > 1 else outs[0]


def qlg_tables():
    init()
    tgx = np.empty(9020, _F32)
    th2x = np.empty(9020, _F32)
    check(lib().m3d_qlg_tables(ptr(tgx), ptr(th2x)), "m3d_qlg_tables")
    return tgx, th2x


def qlg_bot_profile(a, q, vpr, idf):
    init()
    a, q, vpr, idf = (np.ascontiguousarray(x, _F32) for x in (a, q, vpr, idf))
    h = np.empty_like(a)
    check(lib().m3d_qlg_bot_profile(C.c_int(a.size), ptr(a), ptr(q), ptr(vpr), ptr(idf), ptr(h), C.c_uint(0)),
          "m3d_qlg_bot_profile")
    return h


def make_linelist(ll: dict, keep: list) -> LineList:
    """Build an m3d_linelist_t from a dict of arrays (numpy or torch); arrays
    are appended to keep so that they outlive the call."""

    def arr(name, dt):
        if name not in ll or ll[name] is None:
            return None
        a = ll[name]
        if isinstance(a, np.ndarray) or not hasattr(a, "data_ptr"):
            a = np.ascontiguousarray(a, dt)
        keep.append(a)
        return ptr(a)

    s = LineList()
    s.nline = int(len(ll["llam0"]))
    s.llam0 = arr("llam0", np.float64)
    for k in ("lower_ev", "gpref", "grad", "gw1", "gw2", "gstk"):
        setattr(s, k, arr(k, _F32))
    s.unsold = arr("unsold", np.uint8)
    s.lev_i = arr("lev_i", np.int32)
    s.lev_j = arr("lev_j", np.int32)
    s.active = arr("active", np.uint8)
    s.reach_in = arr("reach_in", _F32)
    return s


def line_opacity(ll: dict, llam, chi, eta, cont, logref, cells: dict, dep_mem=None, nlevel=0, do_nlte=False,
                 tol=1e-4, line_reject_frac=0.0, diag=False, one_m_eps=None, chi_scat=None):
    """add_opacity_equi over ncell cells, in place on chi/eta ((ncell, nf) in C order).
    one_m_eps, chi_scat: the line_scattering split (chi_scat accumulated in place).
    Returns (used, strength, reach) with diag, else None."""
    init()
    keep = []
    s = make_linelist(ll, keep)
    nl = s.nline
    dev = _is_dev(chi)
    if dev:
        import torch
        used = torch.zeros(nl, dtype=torch.uint8, device=chi.device) if diag else None
        strength = torch.zeros(nl, dtype=torch.float32, device=chi.device) if diag else None
        reach = torch.zeros(nl, dtype=torch.float32, device=chi.device) if diag else None
    else:
        used = np.zeros(nl, np.uint8) if diag else None
        strength = np.zeros(nl, _F32) if diag else None
        reach = np.zeros(nl, _F32) if diag else None
        llam = np.ascontiguousarray(llam, np.float64)
    nf = int(llam.shape[0])
    ncell = int(chi.shape[0])
    flags = (DEVICE_PTRS if dev else 0) | (LINE_DIAG if diag else 0)
    cf = [cells[k] for k in ("vproj", "inv_df", "vbar2", "e_kT", "lnbase", "ne", "tothi", "stark_pe")]
    if not dev:
        cf = [np.ascontiguousarray(c, _F32) for c in cf]
        cont = np.ascontiguousarray(cont, _F32)
        logref = np.ascontiguousarray(logref, _F32)
        if dep_mem is not None:
            dep_mem = np.ascontiguousarray(dep_mem, _F32)
        if one_m_eps is not None:
            one_m_eps = np.ascontiguousarray(one_m_eps, _F32)
        if chi_scat is not None and (chi_scat.dtype != _F32 or not chi_scat.flags.c_contiguous):
            raise ValueError("chi_scat must be a C-contiguous float32 array (accumulated in place)")
    check(lib().m3d_line_opacity_scat(C.byref(s), C.c_int(nf), ptr(llam), C.c_int(ncell), ptr(chi), ptr(eta),
                                      ptr(cont), ptr(logref), *[ptr(c) for c in cf], ptr(dep_mem), C.c_int(nlevel),
                                      C.c_int(int(do_nlte)), C.c_float(tol), C.c_float(line_reject_frac), ptr(used),
                                      ptr(strength), ptr(reach), ptr(one_m_eps), ptr(chi_scat), C.c_uint(flags)),
          "m3d_line_opacity_scat")
    del keep
    return (used, strength, reach) if diag else None


def chi_scat_units(chi_scat, beta):
    """chi_scat *= 1 - beta in place (add_linelist_opacities, composition_mod.f90:1864-1874)."""
    init()
    dev = _is_dev(chi_scat)
    if not dev:
        if chi_scat.dtype != _F32 or not chi_scat.flags.c_contiguous:
            raise ValueError("chi_scat must be a C-contiguous float32 array (updated in place)")
        beta = np.ascontiguousarray(beta, _F32)
    n = int(np.prod(chi_scat.shape))
    check(lib().m3d_chi_scat_units(C.c_longlong(n), ptr(chi_scat), ptr(beta), C.c_uint(DEVICE_PTRS if dev else 0)),
          "m3d_chi_scat_units")


def lte_background(nu, temp, out=None):
    """beta, Bnu (ncell, nf); device tensors in, device tensors out (nu float64).
    out: (beta, Bnu) device tensors to write into."""
    init()
    if _is_dev(temp):
        import torch
        nu = torch.as_tensor(nu, dtype=torch.float64, device=temp.device).contiguous()
        if out is not None:
            beta, Bnu = out
        else:
            beta = torch.empty((temp.numel(), nu.numel()), dtype=torch.float32, device=temp.device)
            Bnu = torch.empty_like(beta)
        check(lib().m3d_lte_background(C.c_int(nu.numel()), C.c_int(temp.numel()), ptr(nu), ptr(temp), ptr(beta),
                                       ptr(Bnu), C.c_uint(DEVICE_PTRS)), "m3d_lte_background")
        return beta, Bnu
    nu = np.ascontiguousarray(nu, np.float64)
    temp = np.ascontiguousarray(temp, _F32)
    beta = np.empty((temp.size, nu.size), _F32)
    Bnu = np.empty_like(beta)
    check(lib().m3d_lte_background(C.c_int(nu.size), C.c_int(temp.size), ptr(nu), ptr(temp), ptr(beta), ptr(Bnu),
                                   C.c_uint(0)), "m3d_lte_background")
    return beta, Bnu


def work_to_transfer_units(w1, w2, beta, maser_chi_floor=1e-4, suppress_masers=False) -> int:
    init()
    nc, nf = beta.shape
    nfl = C.c_int(0)
    flags = DEVICE_PTRS if _is_dev(w1) else 0
    if flags:
        import torch
        cnt = torch.zeros(1, dtype=torch.int32, device=w1.device)
        check(lib().m3d_work_to_transfer_units(C.c_int(nf), C.c_int(nc), ptr(w1), ptr(w2), ptr(beta),
                                               C.c_double(maser_chi_floor), C.c_int(int(suppress_masers)), ptr(cnt),
                                               C.c_uint(flags)), "m3d_work_to_transfer_units")
        return int(cnt.item())
    check(lib().m3d_work_to_transfer_units(C.c_int(nf), C.c_int(nc), ptr(w1), ptr(w2), ptr(beta),
                                           C.c_double(maser_chi_floor), C.c_int(int(suppress_masers)), C.byref(nfl),
                                           C.c_uint(0)), "m3d_work_to_transfer_units")
    return nfl.value


def formal_solve(solver, slab, work, psi=None, irem=None, escape=None, chi500=None, chi500_up=None, g500=None,
                 eta_row=None, eta_mask=None, rotate=None, extra_flags=0):
    """radiative_transfer of one slab.  rotate = (ds_code(3), bot2pivot, ray_offset(2))
    applies rotate_array first (quadratic solver)."""
    init()
    flags = _flags([work], extra_flags)
    if rotate is not None:
        flags |= ROTATE
        ds_code = (C.c_double * 3)(*rotate[0])
        b2p = float(rotate[1])
        off = (C.c_double * 2)(*(rotate[2] if len(rotate) > 2 else (0.0, 0.0)))
    else:
        ds_code, b2p, off = None, 0.0, None
    check(lib().m3d_formal_solve(C.c_int(solver), C.byref(slab), ptr(work), ptr(psi), ptr(irem), ptr(escape),
                                 ptr(chi500), ptr(chi500_up), ptr(g500), ptr(eta_row), ptr(eta_mask), ds_code,
                                 C.c_double(b2p), off, C.c_uint(flags)), "m3d_formal_solve")


class Hermite(C.Structure):
    """m3d_hermite_t."""

    _fields_ = [(k, C.c_void_p) for k in ("beta", "pe", "dpe_dz", "dlnt_dz", "temp", "hknu", "ghost_pe",
                                           "ghost_dpe_dz", "ghost_dlnt_dz", "ghost_temp")] + [("code_length",
                                                                                               C.c_double)]


def long_char_hermite(slab, work, psi, beta, pe, dpe_dz, dlnt_dz, temp, hknu, ghost=None, code_length=1.0):
    """long_char_hermite (rt_solvers_mod.f90:1052-1504) of one slab, in place on work
    (float32).  ghost: dict pe, dpe_dz, dlnt_dz, temp (ny, nx) of the upstream
    ghost's state, or None for the zeroed top ghost."""
    init()
    dev = _is_dev(work)
    conv = (lambda a: a) if dev else (lambda a: np.ascontiguousarray(a, _F32))
    keep = [conv(a) for a in (beta, pe, dpe_dz, dlnt_dz, temp, hknu)]
    g = [None] * 4 if not ghost else [conv(ghost[k]) for k in ("pe", "dpe_dz", "dlnt_dz", "temp")]
    keep += g
    h = Hermite(*[ptr(a) for a in keep[:6]], *[ptr(a) for a in g], float(code_length))
    check(lib().m3d_long_char_hermite(C.byref(slab), ptr(work), ptr(psi), C.byref(h),
                                      C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_long_char_hermite")
    del keep


def long_char_hermite2(slab, work, psi, pe, dpe_dz, ghost=None, ghost_kind=0, code_length=1.0):
    """long_char_hermite2 (rt_solvers_mod.f90:1536-1895) of one slab, in place on work
    (float32).  ghost: dict pe, dpe_dz (ny, nx) of the upstream ghost, or None for
    the zeroed top ghost; ghost_kind 1 = an upstream neighbour's exit plane,
    2 = the model below the bottom (the default when a ghost is given)."""
    init()
    dev = _is_dev(work)
    conv = (lambda a: a) if dev else (lambda a: np.ascontiguousarray(a, _F32))
    keep = [conv(pe), conv(dpe_dz)]
    g = [None, None] if not ghost else [conv(ghost["pe"]), conv(ghost["dpe_dz"])]
    kind = 0 if not ghost else (ghost_kind or 2)
    check(lib().m3d_long_char_hermite2(C.byref(slab), ptr(work), ptr(psi), ptr(keep[0]), ptr(keep[1]), ptr(g[0]),
                                       ptr(g[1]), C.c_int(kind), C.c_double(code_length),
                                       C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_long_char_hermite2")
    del keep, g


class Hermite3D(C.Structure):
    """m3d_hermite3d_t."""

    _fields_ = [(n, C.c_void_p) for n in ("beta", "pe", "dpe_dx", "dpe_dy", "dpe_dz", "dlnt_dx", "dlnt_dy",
                                          "dlnt_dz", "temp", "hknu")] + [("code_length", C.c_double)]


def short_char_hermite(slab, work, psi, irem, esc, beta, pe, dpe_dx, dpe_dy, dpe_dz, dlnt_dx, dlnt_dy, dlnt_dz,
                       temp, hknu, code_length=1.0):
    """short_char_hermite (rt_solvers_mod.f90:1917-2248) of one slab, in place on
    work (float32); psi, irem, esc (nz, ny, nx, nf) or None as the slab's get_psi
    and split_rates ask."""
    init()
    dev = _is_dev(work)
    conv = (lambda a: a) if dev else (lambda a: np.ascontiguousarray(a, _F32))
    keep = [conv(a) for a in (beta, pe, dpe_dx, dpe_dy, dpe_dz, dlnt_dx, dlnt_dy, dlnt_dz, temp, hknu)]
    h = Hermite3D(*[ptr(a) for a in keep], float(code_length))
    check(lib().m3d_short_char_hermite(C.byref(slab), ptr(work), ptr(psi), ptr(irem), ptr(esc), C.byref(h),
                                       C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_short_char_hermite")
    del keep


def rotate_array(slab, work, ds_code, bot2pivot, ray_offset=(0.0, 0.0)):
    init()
    check(lib().m3d_rotate_array(C.byref(slab), ptr(work), (C.c_double * 3)(*ds_code), C.c_double(bot2pivot),
                                 (C.c_double * 2)(*ray_offset), C.c_uint(_flags([work]))), "m3d_rotate_array")


def upstream_boundary(slab, work, mode, mem=None, ds3_code=1.0, ghost_r500=None, ghost_temp=None, nu=None):
    init()
    check(lib().m3d_upstream_boundary(C.byref(slab), ptr(work), C.c_int(mode), ptr(mem), C.c_float(ds3_code),
                                      ptr(ghost_r500), ptr(ghost_temp), ptr(nu), C.c_uint(_flags([work]))),
          "m3d_upstream_boundary")


def integrate_intensity(wmu, inu, psi, Jnu, PsiJ):
    init()
    check(lib().m3d_integrate_intensity(C.c_int(int(np.prod(inu.shape))), C.c_float(wmu), ptr(inu), ptr(psi),
                                        ptr(Jnu), ptr(PsiJ), C.c_uint(_flags([inu]))), "m3d_integrate_intensity")


def _atmos(atm: dict, keep: list) -> Atmos:
    """m3d_atmos_t of an atmosphere dict (numpy host arrays or torch CUDA tensors)."""
    a = Atmos()
    a.nx, a.ny, a.nz = atm["nx"], atm["ny"], atm["nz"]
    slab_nz = np.ascontiguousarray(atm.get("slab_nz", [atm["nz"]]), np.int32)
    keep.append(slab_nz)
    a.nslab = slab_nz.size
    a.slab_nz = ptr(slab_nz)
    a.ds_cm[:] = list(atm.get("ds_cm", (1.0, 1.0, 1.0)))
    a.ds_code[:] = list(atm.get("ds_code", (1.0, 1.0, 1.0)))
    a.pivot_z = float(atm.get("pivot_z", 0.0))
    a.ray_offset[:] = list(atm.get("ray_offset", (0.0, 0.0)))

    def fld(x):
        if isinstance(x, np.ndarray):
            x = np.ascontiguousarray(x, _F32)
        keep.append(x)
        return ptr(x)

    for k in ("temp", "chi_c", "vx", "vy", "vz", "e_kT", "ne", "tothi", "stark_pe"):
        setattr(a, k, fld(atm[k]))
    sp_list = atm["species"]
    sarr = (Species * max(1, len(sp_list)))()
    for i, sp in enumerate(sp_list):
        sarr[i].ll = make_linelist(sp, keep)
        sarr[i].inv_df = fld(sp["inv_df"])
        sarr[i].vbar2 = fld(sp["vbar2"])
        sarr[i].lnbase = fld(sp["lnbase"])
    keep.append(sarr)
    a.nspecies = len(sp_list)
    a.species = C.cast(sarr, C.c_void_p)
    a.tol = atm.get("tol", 1e-4)
    a.maser_chi_floor = atm.get("maser_chi_floor", 1e-4)
    a.maser_dtau_max = atm.get("maser_dtau_max", 2.0)
    a.maser_Inu_max = atm.get("maser_Inu_max", 1e30)
    return a


def lte_synthesis(atm: dict, nu, llam, vec, wmu, fp64=False, return_itop=False, device=False):
    """The LTE output pass of one frequency window for every ray (m3d_lte_synthesis).

    atm: dict with nx, ny, nz, slab_nz, ds_cm, ds_code, pivot_z, ray_offset and the
    per-cell fields (numpy for host buffers, torch CUDA tensors with device=True),
    species: list of dicts (linelist arrays + inv_df, vbar2, lnbase).
    Returns (ie (nray, nf), flux (nf,), i_top or None)."""
    init()
    keep = []
    a = _atmos(atm, keep)
    vec = np.ascontiguousarray(vec, np.float64)
    wmu = np.ascontiguousarray(wmu, np.float64)
    nray = wmu.size
    nf = int(nu.shape[0])
    flags = (FP64 if fp64 else 0) | (DEVICE_PTRS if device else 0)
    if device:
        import torch
        dev = atm["temp"].device
        ie = torch.empty((nray, nf), dtype=torch.float32, device=dev)
        flux = torch.empty(nf, dtype=torch.float32, device=dev)
        itop = torch.empty((nray, a.ny, a.nx, nf), dtype=torch.float64 if fp64 else torch.float32,
                           device=dev) if return_itop else None
    else:
        nu = np.ascontiguousarray(nu, np.float64)
        llam = np.ascontiguousarray(llam, np.float64)
        ie = np.empty((nray, nf), _F32)
        flux = np.empty(nf, _F32)
        itop = np.empty((nray, a.ny, a.nx, nf), np.float64 if fp64 else _F32) if return_itop else None
    check(lib().m3d_lte_synthesis(C.byref(a), C.c_int(nf), ptr(nu), ptr(llam), C.c_int(nray), ptr(vec), ptr(wmu),
                                  ptr(itop), ptr(ie), ptr(flux), C.c_uint(flags)), "m3d_lte_synthesis")
    del keep
    return ie, flux, itop


def lte_synthesis_windows(atm: dict, nu, llam, vec, wmu, fp64=False, return_itop=False, device=False):
    """lte_synthesis over a batch of windows of 32 frequencies in one call
    (m3d_lte_synthesis_windows): nu and llam (nwin, 32).  Returns (ie (nray, nwin 32),
    flux (nwin 32,), i_top or None), equal bit for bit to one lte_synthesis per
    window, the windows' outputs one after the other."""
    init()
    keep = []
    a = _atmos(atm, keep)
    vec = np.ascontiguousarray(vec, np.float64)
    wmu = np.ascontiguousarray(wmu, np.float64)
    nray = wmu.size
    nwin, nf = int(nu.shape[0]), int(nu.shape[1])
    nft = nwin * nf
    flags = (FP64 if fp64 else 0) | (DEVICE_PTRS if device else 0)
    if device:
        import torch
        dev = atm["temp"].device
        nu, llam = nu.contiguous(), llam.contiguous()
        ie = torch.empty((nray, nft), dtype=torch.float32, device=dev)
        flux = torch.empty(nft, dtype=torch.float32, device=dev)
        itop = torch.empty((nray, a.ny, a.nx, nft), dtype=torch.float64 if fp64 else torch.float32,
                           device=dev) if return_itop else None
    else:
        nu = np.ascontiguousarray(nu, np.float64)
        llam = np.ascontiguousarray(llam, np.float64)
        ie = np.empty((nray, nft), _F32)
        flux = np.empty(nft, _F32)
        itop = np.empty((nray, a.ny, a.nx, nft), np.float64 if fp64 else _F32) if return_itop else None
    check(lib().m3d_lte_synthesis_windows(C.byref(a), C.c_int(nwin), C.c_int(nf), ptr(nu), ptr(llam), C.c_int(nray),
                                          ptr(vec), ptr(wmu), ptr(itop), ptr(ie), ptr(flux), C.c_uint(flags)),
          "m3d_lte_synthesis_windows")
    del keep
    return ie, flux, itop


def lte_transfer_units(atm: dict, nu, llam, vec, fp64=False, device=False, out=None):
    """The opacity stage of the LTE pass for one direction (m3d_lte_transfer_units):
    (chi, S), each (ncell, nf), float32 (float64 with fp64).  out: preallocated
    (chi, S) to write into."""
    init()
    keep = []
    a = _atmos(atm, keep)
    vec = np.ascontiguousarray(vec, np.float64).reshape(3)
    nf = int(nu.shape[0])
    ncell = a.nx * a.ny * a.nz
    flags = (FP64 if fp64 else 0) | (DEVICE_PTRS if device else 0)
    if out is not None:
        chi, S = out
    elif device:
        import torch
        dt = torch.float64 if fp64 else torch.float32
        chi = torch.empty((ncell, nf), dtype=dt, device=atm["temp"].device)
        S = torch.empty_like(chi)
    else:
        nu = np.ascontiguousarray(nu, np.float64)
        llam = np.ascontiguousarray(llam, np.float64)
        chi = np.empty((ncell, nf), np.float64 if fp64 else _F32)
        S = np.empty_like(chi)
    if device:
        order_after_torch(chi)
    check(lib().m3d_lte_transfer_units(C.byref(a), C.c_int(nf), ptr(nu), ptr(llam), ptr(vec), ptr(chi), ptr(S),
                                       C.c_uint(flags)), "m3d_lte_transfer_units")
    del keep
    return chi, S


class LteGrad(C.Structure):
    """m3d_lte_grad_t."""

    _fields_ = [(k, C.c_void_p) for k in ("temp", "chi_c", "e_kT", "inv_df", "lnbase", "gpref")]


def lte_synthesis_adjoint(atm: dict, nu, llam, vec, wmu, g_flux, device=False, grads=None):
    """The reverse mode of lte_synthesis for one window of 32 frequencies
    (m3d_lte_synthesis_adjoint): given g_flux = dL/dflux (nf,), returns the dict of
    dL/d(input): temp, chi_c, e_kT (ncell,), inv_df, lnbase (nspecies, ncell), gpref
    (all lines, species in order).  grads: arrays to accumulate into (else zeros)."""
    init()
    keep = []
    a = _atmos(atm, keep)
    vec = np.ascontiguousarray(vec, np.float64)
    wmu = np.ascontiguousarray(wmu, np.float64)
    nray = wmu.size
    nf = int(nu.shape[0])
    ncell = a.nx * a.ny * a.nz
    nsp = len(atm["species"])
    nline = sum(len(sp["llam0"]) for sp in atm["species"])
    if grads is None:
        if device:
            import torch
            dev = atm["temp"].device
            z = lambda *shape: torch.zeros(shape, dtype=torch.float32, device=dev)
        else:
            z = lambda *shape: np.zeros(shape, _F32)
        grads = {"temp": z(ncell), "chi_c": z(ncell), "e_kT": z(ncell), "inv_df": z(max(nsp, 1), ncell),
                 "lnbase": z(max(nsp, 1), ncell), "gpref": z(max(nline, 1))}
    if not device:
        nu = np.ascontiguousarray(nu, np.float64)
        llam = np.ascontiguousarray(llam, np.float64)
        g_flux = np.ascontiguousarray(g_flux, _F32)
    else:
        order_after_torch(grads["temp"])
    g = LteGrad(*[ptr(grads[k]) for k in ("temp", "chi_c", "e_kT", "inv_df", "lnbase", "gpref")])
    flags = DEVICE_PTRS if device else 0
    check(lib().m3d_lte_synthesis_adjoint(C.byref(a), C.c_int(nf), ptr(nu), ptr(llam), C.c_int(nray), ptr(vec),
                                          ptr(wmu), ptr(g_flux), C.byref(g), C.c_uint(flags)),
          "m3d_lte_synthesis_adjoint")
    del keep
    return grads


def hop_set_state(atm: dict):
    """m3d_hop_set_state: load a state (host arrays) for hop_opacity."""
    init()
    keep = []
    a = _atmos(atm, keep)
    check(lib().m3d_hop_set_state(C.byref(a)), "m3d_hop_set_state")
    del keep


def hop_opacity(lam, chi, scat, include_absmet=0, include_llist=1, line_margin=10.0, line_scat=-1):
    """m3d_hop_opacity with libhop's hop_opacity arguments: adds the loaded state's
    line list to chi (nlam, n) float32 in place (wavelength fastest per cell)."""
    init()
    lam = np.ascontiguousarray(lam, np.float64)
    assert chi.dtype == np.float32 and chi.flags.c_contiguous and scat.dtype == np.float32
    check(lib().m3d_hop_opacity(C.c_int(lam.size), ptr(lam), ptr(chi), ptr(scat), C.c_int(include_absmet),
                                C.c_int(include_llist), C.c_double(line_margin), C.c_int(line_scat)),
          "m3d_hop_opacity")


def eta_spread(vecs, ds, dz_upstream=None, one_dimensional=False) -> tuple[int, int]:
    """eta_rx, eta_ry of update_eta_mask (rt_patch_mod.f90:3683-3700): the horizontal
    reach of an upwind point over the slab's directions, plus the cell beyond it."""
    if one_dimensional:
        return 0, 0
    dz = ds[2] if dz_upstream is None else max(ds[2], dz_upstream)
    sx = max(abs(v[0] / v[2]) for v in vecs)
    sy = max(abs(v[1] / v[2]) for v in vecs)
    return int(np.floor(sx * dz / ds[0])) + 1, int(np.floor(sy * dz / ds[1])) + 1


def update_eta_mask(slab, work, beta, eta_src, eta_mask, rx, ry, eta_gsrc=None):
    """update_eta_mask with dense flags (uint8), in place; eta_gsrc given = test the ghost plane."""
    init()
    ghost = eta_gsrc is not None
    check(lib().m3d_update_eta_mask(C.byref(slab), ptr(work), ptr(beta), ptr(eta_src), ptr(eta_gsrc), ptr(eta_mask),
                                    C.c_int(rx), C.c_int(ry), C.c_int(int(ghost)),
                                    C.c_uint(_flags([work, beta, eta_src]) & DEVICE_PTRS)), "m3d_update_eta_mask")


def lte_populations(atom: dict, temp, lsaha, totn, dxi=None):
    """compute_lte_populations (level partition function): returns nstar (nlevel, ncell); totn updated in place."""
    init()
    from .stateq import make_atom
    st, keep = make_atom(atom)
    temp, lsaha = np.ascontiguousarray(temp, _F32), np.ascontiguousarray(lsaha, _F32)
    dxi = None if dxi is None else np.ascontiguousarray(dxi, _F32)
    if totn.dtype != np.float64 or not totn.flags.c_contiguous:
        raise ValueError("totn must be a C-contiguous float64 array (updated in place)")
    nstar = np.zeros((st.nlevel, temp.size), np.float64)
    check(lib().m3d_lte_populations(C.byref(st), C.c_int(temp.size), ptr(temp), ptr(lsaha), ptr(dxi), ptr(nstar),
                                    ptr(totn), C.c_uint(0)), "m3d_lte_populations")
    return nstar


def particle_fields(awgt, vmic, iso_frac, temp, n, part, population_scale=0.0):
    """inverse_doppler_factor, compute_vbar2 and lnbase of one isotope: (inv_df, vbar2, lnbase)."""
    init()
    temp = np.ascontiguousarray(temp, _F32)
    n, part = np.ascontiguousarray(n, np.float64), np.ascontiguousarray(part, np.float64)
    idf, vb, lb = (np.zeros(temp.size, _F32) for _ in range(3))
    check(lib().m3d_particle_fields(C.c_int(temp.size), C.c_double(awgt), C.c_float(vmic), C.c_double(iso_frac),
                                    C.c_double(population_scale), ptr(temp), ptr(n), ptr(part), ptr(idf), ptr(vb),
                                    ptr(lb), C.c_uint(0)), "m3d_particle_fields")
    return idf, vb, lb


def lte_emission(chi_cont, Bnu, beta, sigma=None, Jnu=None, jnu_init=0, PsiJ=None, Jali=None, jali_valid=False,
                 scat_op_max=0.9, out=None):
    """lte_background_emission + convert_to_work_units: (xhat, ehat, dJnu, n_negative).

    jnu_init: 0 Jnu given, 1 Jnu = Bnu (the Planck start), 2 Jnu = 0; PsiJ given:
    the OAB step with Jali (in/out).  out: optional (xhat, ehat, dJnu) arrays."""
    init()
    dev = _is_dev(Bnu)
    if out is None:
        if dev:
            import torch
            out = tuple(torch.empty_like(Bnu) for _ in range(3))
        else:
            out = tuple(np.empty(np.shape(Bnu), _F32) for _ in range(3))
    xhat, ehat, dj = out
    if not dev:
        chi_cont, Bnu, beta, sigma, Jnu, PsiJ = (None if a is None else np.ascontiguousarray(a, _F32)
                                                 for a in (chi_cont, Bnu, beta, sigma, Jnu, PsiJ))
    nf, ncell = int(Bnu.shape[-1]), int(np.prod(Bnu.shape[:-1]))
    neg = C.c_longlong()
    check(lib().m3d_lte_emission(C.c_int(nf), C.c_int(ncell), ptr(chi_cont), ptr(sigma), ptr(Bnu), ptr(beta),
                                 ptr(Jnu), C.c_int(jnu_init), ptr(PsiJ), ptr(Jali), C.c_int(int(jali_valid)),
                                 C.c_double(scat_op_max), ptr(xhat), ptr(ehat), ptr(dj), C.byref(neg),
                                 C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_lte_emission")
    return xhat, ehat, dj, neg.value

"""Model-atom opacities and ALI rate integrals of one frequency window over
libm3dgpu.so (include/m3dgpu.h, m3d_bb_opacity and friends).

A window is a dict of numpy arrays (dispatch_b200.synth.atom_window builds
one) with the fields of m3d_atom_window_t.  Per-point arrays (nf, ncell) are
numpy arrays of shape (ncell, nf) in C order (frequency fastest) or CUDA
tensors; per-cell level arrays are (nlevel, ncell) (cell fastest).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DEVICE_PTRS, M3DError, check, init, lib, order_after_torch, ptr

_P = C.c_void_p


class AtomWindow(C.Structure):
    """m3d_atom_window_t."""

    _fields_ = [("nf", C.c_int), ("nline", C.c_int), ("ncont", C.c_int), ("nlevel", C.c_int),
                ("line_i", _P), ("line_j", _P), ("line_ntrans", _P), ("line_index", _P),
                ("line_blue", _P), ("line_red", _P), ("line_off", _P),
                ("q", _P), ("wnu", _P), ("wq", _P), ("Bij", _P), ("Aij", _P), ("lower_ev", _P),
                ("line_active", _P), ("sums_over_windows", _P),
                ("grad", _P), ("gw1", _P), ("gw2", _P), ("gstk", _P), ("unsold", _P),
                ("cont_i", _P), ("cont_j", _P), ("cont_ntrans", _P), ("cont_blue", _P), ("cont_red", _P),
                ("cont_off", _P), ("alpha", _P), ("cwnu", _P), ("cont_active", _P),
                ("g", _P), ("ev", _P), ("cut_x", C.c_double)]


class RateOpts(C.Structure):
    """m3d_rate_opts_t."""

    _fields_ = [("split_rates", C.c_int), ("preconditioning", C.c_int), ("per_direction", C.c_int),
                ("use_flags", C.c_int), ("do_scat", C.c_int), ("nwords", C.c_int),
                ("wmu", C.c_float), ("wtot", C.c_float)]


_KINDS = {"line_i": np.int32, "line_j": np.int32, "line_ntrans": np.int32, "line_index": np.int32,
          "line_blue": np.int32, "line_red": np.int32, "line_off": np.int32, "q": np.float32,
          "wnu": np.float64, "wq": np.float64, "Bij": np.float64, "Aij": np.float64, "lower_ev": np.float64,
          "line_active": np.uint8, "sums_over_windows": np.uint8, "grad": np.float64, "gw1": np.float64,
          "gw2": np.float64, "gstk": np.float64, "unsold": np.uint8, "cont_i": np.int32, "cont_j": np.int32,
          "cont_ntrans": np.int32, "cont_blue": np.int32, "cont_red": np.int32, "cont_off": np.int32,
          "alpha": np.float32, "cwnu": np.float64, "cont_active": np.uint8, "g": np.float64, "ev": np.float64}


def make_window(win: dict) -> tuple[AtomWindow, list]:
    """The m3d_atom_window_t of a window dict, and the arrays it points into."""
    keep = []
    s = AtomWindow()
    s.nf, s.nline, s.ncont, s.nlevel = int(win["nf"]), int(win["nline"]), int(win["ncont"]), int(win["nlevel"])
    for k, dt in _KINDS.items():
        v = win.get(k)
        if v is None:
            setattr(s, k, None)
            continue
        a = np.ascontiguousarray(v, dt)
        keep.append(a)
        setattr(s, k, a.ctypes.data)
    s.cut_x = float(win.get("cut_x", 70.0))
    return s, keep


def _flags(*arrays) -> int:
    for a in arrays:
        if a is not None and not isinstance(a, np.ndarray):
            order_after_torch(a)
            return DEVICE_PTRS
    return 0


def _c(a, dt):
    if a is None or not isinstance(a, np.ndarray):
        return a
    return np.ascontiguousarray(a, dt)


def _inplace(a, dt, name):
    if isinstance(a, np.ndarray) and (a.dtype != dt or not a.flags.c_contiguous):
        raise M3DError(f"{name} must be a C-contiguous {np.dtype(dt).name} array (updated in place)")
    return a


def _ncell(a) -> int:
    return int(a.shape[-1])


def bb_damping(win, ne, tothi, vbar2, stark_pe, unsold, inv_df, out=None):
    """adamp (nline, ncell) of bound_bound_damping."""
    init()
    st, keep = make_window(win)
    args = [_c(x, np.float32) for x in (ne, tothi, vbar2, stark_pe, unsold, inv_df)]
    n = _ncell(args[-1])
    if out is None:
        out = np.zeros((st.nline, n), np.float32)
    check(lib().m3d_bb_damping(C.byref(st), C.c_int(n), *[ptr(a) for a in args], ptr(out),
                               C.c_uint(_flags(*args, out))), "m3d_bb_damping")
    return out


def bf_opacity(win, b, nstar, pop_ratio, e_kT, xhat, ehat):
    """add_bound_free_opacities into xhat, ehat (ncell, nf) float32 in place."""
    init()
    st, keep = make_window(win)
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    _inplace(xhat, np.float32, "xhat")
    _inplace(ehat, np.float32, "ehat")
    n = _ncell(pop_ratio)
    check(lib().m3d_bf_opacity(C.byref(st), C.c_int(n), ptr(b), ptr(nstar), ptr(pop_ratio), ptr(e_kT), ptr(xhat),
                               ptr(ehat), C.c_uint(_flags(nstar, xhat))), "m3d_bf_opacity")


def bb_opacity(win, b, nstar, pop_ratio, e_kT, inv_df, vproj, adamp, xhat, ehat, lte=False, wmu=0.0,
               split=None, wphi=None):
    """add_bound_bound_opacities of one direction into xhat, ehat in place.

    split: None, or a dict with opac_L, opac_R, id, chi_L, chi_R, chi_id arrays
    (ncell, nf) that receive the tracking; wphi: None or (nline_atom, ncell)."""
    init()
    st, keep = make_window(win)
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    inv_df, vproj, adamp = (_c(x, np.float32) for x in (inv_df, vproj, adamp))
    _inplace(xhat, np.float32, "xhat")
    _inplace(ehat, np.float32, "ehat")
    s = [None] * 6
    if split is not None:
        s = [split[k] for k in ("opac_L", "opac_R", "id", "chi_L", "chi_R", "chi_id")]
    n = _ncell(pop_ratio)
    check(lib().m3d_bb_opacity(C.byref(st), C.c_int(n), ptr(b), ptr(nstar), ptr(pop_ratio), ptr(e_kT), ptr(inv_df),
                               ptr(vproj), ptr(adamp), C.c_int(int(lte)), C.c_float(wmu), ptr(xhat), ptr(ehat),
                               *[ptr(a) for a in s], ptr(wphi), C.c_uint(_flags(nstar, xhat))), "m3d_bb_opacity")


def bb_opacity_units(win, b, nstar, pop_ratio, e_kT, inv_df, vproj, adamp, xhat, ehat, beta, chi, S, split,
                     wmu=0.0, wphi=None, maser_chi_floor=1e-4):
    """bb_opacity (non-LTE, split tracking into split) and transfer_units_split of one
    direction in one pass (m3d_bb_opacity_units): the background xhat, ehat is read,
    chi and S receive the transfer units."""
    init()
    st, keep = make_window(win)
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    inv_df, vproj, adamp, xhat, ehat, beta = (_c(x, np.float32) for x in (inv_df, vproj, adamp, xhat, ehat, beta))
    _inplace(chi, np.float32, "chi")
    _inplace(S, np.float32, "S")
    s = [split[k] for k in ("opac_L", "opac_R", "id", "chi_L", "chi_R", "chi_id")]
    n = _ncell(pop_ratio)
    check(lib().m3d_bb_opacity_units(C.byref(st), C.c_int(n), ptr(b), ptr(nstar), ptr(pop_ratio), ptr(e_kT),
                                     ptr(inv_df), ptr(vproj), ptr(adamp), C.c_float(wmu), ptr(xhat), ptr(ehat),
                                     ptr(beta), C.c_double(maser_chi_floor), ptr(chi), ptr(S),
                                     *[ptr(a) for a in s], ptr(wphi), C.c_uint(_flags(nstar, chi))),
          "m3d_bb_opacity_units")


def new_split(ncell: int, nf: int) -> dict:
    z = lambda dt: np.zeros((ncell, nf), dt)
    return {"opac_L": z(np.float32), "opac_R": z(np.float32), "id": z(np.int32),
            "chi_L": z(np.float32), "chi_R": z(np.float32), "chi_id": z(np.int32)}


def transfer_units_split(w1, w2, beta, split, scat=None, maser_chi_floor=1e-4, suppress_masers=False) -> int:
    """work_to_transfer_units with split rates, in place; returns the floored count."""
    init()
    _inplace(w1, np.float32, "w1")
    _inplace(w2, np.float32, "w2")
    beta, scat = _c(beta, np.float32), _c(scat, np.float32)
    ncell, nf = int(w1.shape[0]), int(w1.shape[1])
    nfl = C.c_int()
    check(lib().m3d_work_to_transfer_units_split(C.c_int(nf), C.c_int(ncell), ptr(w1), ptr(w2), ptr(beta),
                                                 ptr(split["opac_L"]), ptr(split["opac_R"]), ptr(scat),
                                                 C.c_double(maser_chi_floor), C.c_int(int(suppress_masers)),
                                                 C.byref(nfl), C.c_uint(_flags(w1, beta))),
          "m3d_work_to_transfer_units_split")
    return nfl.value


def bb_rates(win, b, nstar, pop_ratio, e_kT, inv_df, vproj, adamp, inu, beta, Bnu, gamma_ij, gamma_ji,
             work1=None, psi=None, irem=None, escape=None, split=None, scat=None, flags_in=None,
             flags_raise=None, split_rates=True, preconditioning=True, per_direction=True, wmu=1.0, wtot=1.0):
    """bound_bound_rates of one direction; gamma_ij/ji (nline + ncont, ncell) accumulated in place."""
    init()
    st, keep = make_window(win)
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    f32 = [_c(x, np.float32) for x in (inv_df, vproj, adamp, work1, inu, psi, irem, escape, beta, Bnu, scat)]
    inv_df, vproj, adamp, work1, inu, psi, irem, escape, beta, Bnu, scat = f32
    _inplace(gamma_ij, np.float32, "gamma_ij")
    _inplace(gamma_ji, np.float32, "gamma_ji")
    s = [None] * 6
    if split is not None:
        s = [split[k] for k in ("opac_L", "opac_R", "id", "chi_L", "chi_R", "chi_id")]
    use_flags = flags_in is not None
    nwords = int(flags_in.shape[0]) if use_flags else 0
    o = RateOpts(int(split_rates), int(preconditioning), int(per_direction), int(use_flags), int(scat is not None),
                 nwords, float(wmu), float(wtot))
    n = _ncell(pop_ratio)
    check(lib().m3d_bb_rates(C.byref(st), C.byref(o), C.c_int(n), ptr(b), ptr(nstar), ptr(pop_ratio), ptr(e_kT),
                             ptr(inv_df), ptr(vproj), ptr(adamp), ptr(work1), ptr(inu), ptr(psi), ptr(irem),
                             ptr(escape), ptr(beta), ptr(Bnu), *[ptr(a) for a in s], ptr(scat), ptr(flags_in),
                             ptr(flags_raise), ptr(gamma_ij), ptr(gamma_ji), C.c_uint(_flags(nstar, inu))),
          "m3d_bb_rates")


def bf_rates(win, b, nstar, e_kT, Jnu, PsiJ, beta, gamma_ij, gamma_ji, preconditioning=True):
    """bound_free_rates from the angle-integrated Jnu and PsiJ; gamma accumulated in place."""
    init()
    st, keep = make_window(win)
    b, nstar, e_kT = (_c(x, np.float64) for x in (b, nstar, e_kT))
    two = np.ascontiguousarray(win["twohnu3_c2"], np.float32)
    if not isinstance(Jnu, np.ndarray):
        import torch
        two = torch.from_numpy(two).to(Jnu.device)
    Jnu, PsiJ, beta = (_c(x, np.float32) for x in (Jnu, PsiJ, beta))
    _inplace(gamma_ij, np.float32, "gamma_ij")
    _inplace(gamma_ji, np.float32, "gamma_ji")
    n = _ncell(e_kT)
    check(lib().m3d_bf_rates(C.byref(st), C.c_int(n), C.c_int(int(preconditioning)), ptr(b), ptr(nstar), ptr(e_kT),
                             ptr(two), ptr(Jnu), ptr(PsiJ), ptr(beta), ptr(gamma_ij), ptr(gamma_ji),
                             C.c_uint(_flags(nstar, Jnu))), "m3d_bf_rates")


def integrate_rates(win, gw_ij, gw_ji, gamma_ij, gamma_ji):
    """The window's rate sums into the atom's (nrad, ncell) rates by transition index."""
    init()
    st, keep = make_window(win)
    gw_ij, gw_ji = _c(gw_ij, np.float32), _c(gw_ji, np.float32)
    _inplace(gamma_ij, np.float32, "gamma_ij")
    _inplace(gamma_ji, np.float32, "gamma_ji")
    n = _ncell(gw_ij)
    check(lib().m3d_integrate_rates(C.byref(st), C.c_int(n), ptr(gw_ij), ptr(gw_ji), ptr(gamma_ij), ptr(gamma_ji),
                                    C.c_uint(_flags(gw_ij, gamma_ij))), "m3d_integrate_rates")


def normalize_profiles(atom: dict, nstar, wphi, gamma_ij, gamma_ji, has_wphi, first_iter: bool):
    """normalize_profiles on the atom's (nrad, ncell) rates, in place."""
    init()
    ti = np.ascontiguousarray(atom["ti"], np.int32)
    tj = np.ascontiguousarray(atom["tj"], np.int32)
    act = None if atom.get("active") is None else np.ascontiguousarray(atom["active"], np.uint8)
    hw = np.ascontiguousarray(has_wphi, np.uint8)
    nstar = _c(nstar, np.float64)
    n = _ncell(gamma_ij)
    check(lib().m3d_normalize_profiles(C.c_int(n), C.c_int(int(atom["nline"])), C.c_int(len(ti)),
                                       C.c_void_p(ti.ctypes.data), C.c_void_p(tj.ctypes.data),
                                       None if act is None else C.c_void_p(act.ctypes.data),
                                       C.c_void_p(hw.ctypes.data), C.c_int(int(first_iter)), ptr(nstar), ptr(wphi),
                                       ptr(gamma_ij), ptr(gamma_ji), C.c_uint(_flags(nstar, gamma_ij))),
          "m3d_normalize_profiles")


def combine_twins(a, b):
    """a = b = (a + b)/2 in place (float32)."""
    init()
    _inplace(a, np.float32, "a")
    _inplace(b, np.float32, "b")
    n = int(a.size if isinstance(a, np.ndarray) else a.numel())
    check(lib().m3d_combine_twins(C.c_longlong(n), ptr(a), ptr(b), C.c_uint(_flags(a, b))), "m3d_combine_twins")

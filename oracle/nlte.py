"""ctypes front end of the model-atom opacity and rate oracle (oracle/or_nlte.c).

TEST INFRASTRUCTURE ONLY: the checker of the NLTE kernels.  Windows and arrays
have the layout of dispatch_b200.nlte.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import lib, qlg_tables

_P = C.c_void_p

_FIELDS = [("li", "line_i", np.int32), ("lj", "line_j", np.int32), ("lntrans", "line_ntrans", np.int32),
           ("lindex", "line_index", np.int32), ("lblue", "line_blue", np.int32), ("lred", "line_red", np.int32),
           ("loff", "line_off", np.int32), ("q", "q", np.float32), ("wnu", "wnu", np.float64),
           ("wq", "wq", np.float64), ("Bij", "Bij", np.float64), ("Aij", "Aij", np.float64),
           ("lower_ev", "lower_ev", np.float64), ("lactive", "line_active", np.uint8),
           ("lsums", "sums_over_windows", np.uint8), ("grad", "grad", np.float64), ("gw1", "gw1", np.float64),
           ("gw2", "gw2", np.float64), ("gstk", "gstk", np.float64), ("unsold", "unsold", np.uint8),
           ("ci", "cont_i", np.int32), ("cj", "cont_j", np.int32), ("cntrans", "cont_ntrans", np.int32),
           ("cblue", "cont_blue", np.int32), ("cred", "cont_red", np.int32), ("coff", "cont_off", np.int32),
           ("alpha", "alpha", np.float32), ("cwnu", "cwnu", np.float64), ("cactive", "cont_active", np.uint8),
           ("g", "g", np.float64), ("ev", "ev", np.float64)]


class NlWindow(C.Structure):
    _fields_ = ([("nf", C.c_int), ("nline", C.c_int), ("ncont", C.c_int), ("nlevel", C.c_int)]
                + [(n, _P) for n, _, _ in _FIELDS] + [("cut_x", C.c_double)])


class NlRateOpts(C.Structure):
    _fields_ = [("split", C.c_int), ("precond", C.c_int), ("per_direction", C.c_int), ("use_flags", C.c_int),
                ("do_scat", C.c_int), ("pad", C.c_int), ("wmu", C.c_float), ("wtot", C.c_float)]


def make_window(win: dict):
    keep = []
    s = NlWindow()
    s.nf, s.nline, s.ncont, s.nlevel = int(win["nf"]), int(win["nline"]), int(win["ncont"]), int(win["nlevel"])
    for name, key, dt in _FIELDS:
        v = win.get(key)
        if v is None:
            setattr(s, name, None)
            continue
        a = np.ascontiguousarray(v, dt)
        keep.append(a)
        setattr(s, name, a.ctypes.data)
    s.cut_x = float(win.get("cut_x", 70.0))
    return s, keep


def _vp(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dt)


_tab = None


def _tables():
    global _tab
    if _tab is None:
        _tab = tuple(np.ascontiguousarray(t, np.float32) for t in qlg_tables())
    return _tab


def bb_damping(win, ne, tothi, vbar2, stark_pe, unsold, inv_df):
    st, keep = make_window(win)
    args = [_c(x, np.float32) for x in (ne, tothi, vbar2, stark_pe, unsold, inv_df)]
    out = np.zeros((st.nline, args[-1].size), np.float32)
    lib().or_bb_damping(C.byref(st), C.c_int(args[-1].size), *[_vp(a) for a in args], _vp(out))
    return out


def bf_opacity(win, b, nstar, pop_ratio, e_kT, xhat, ehat):
    st, keep = make_window(win)
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    assert xhat.dtype == np.float32 and ehat.dtype == np.float32 and xhat.flags.c_contiguous
    lib().or_bf_opacity(C.byref(st), C.c_int(pop_ratio.size), _vp(b), _vp(nstar), _vp(pop_ratio), _vp(e_kT),
                        _vp(xhat), _vp(ehat))


def bb_opacity(win, b, nstar, pop_ratio, e_kT, inv_df, vproj, adamp, xhat, ehat, lte=False, wmu=0.0,
               split=None, wphi=None):
    st, keep = make_window(win)
    tgx, th2x = _tables()
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    inv_df, vproj, adamp = (_c(x, np.float32) for x in (inv_df, vproj, adamp))
    s = [None] * 6
    if split is not None:
        s = [split[k] for k in ("opac_L", "opac_R", "id", "chi_L", "chi_R", "chi_id")]
    lib().or_bb_opacity(C.byref(st), C.c_int(pop_ratio.size), _vp(b), _vp(nstar), _vp(pop_ratio), _vp(e_kT),
                        _vp(inv_df), _vp(vproj), _vp(adamp), _vp(tgx), _vp(th2x), C.c_int(int(lte)),
                        C.c_int(int(split is not None)), C.c_float(wmu), _vp(xhat), _vp(ehat),
                        *[_vp(a) for a in s], _vp(wphi))


def transfer_units_split(w1, w2, beta, split, scat=None, maser_chi_floor=1e-4, suppress_masers=False):
    beta, scat = _c(beta, np.float32), _c(scat, np.float32)
    f = lib().or_transfer_units_split
    return f(C.c_int(w1.shape[1]), C.c_int(w1.shape[0]), _vp(w1), _vp(w2), _vp(beta), _vp(split["opac_L"]),
             _vp(split["opac_R"]), _vp(scat), C.c_double(maser_chi_floor), C.c_int(int(suppress_masers)))


def bb_rates(win, b, nstar, pop_ratio, e_kT, inv_df, vproj, adamp, inu, beta, Bnu, gamma_ij, gamma_ji,
             work1=None, psi=None, irem=None, escape=None, split=None, scat=None, flags_in=None,
             flags_raise=None, split_rates=True, preconditioning=True, per_direction=True, wmu=1.0, wtot=1.0):
    st, keep = make_window(win)
    tgx, th2x = _tables()
    b, nstar, pop_ratio, e_kT = (_c(x, np.float64) for x in (b, nstar, pop_ratio, e_kT))
    f32 = [_c(x, np.float32) for x in (inv_df, vproj, adamp, work1, inu, psi, irem, escape, beta, Bnu, scat)]
    inv_df, vproj, adamp, work1, inu, psi, irem, escape, beta, Bnu, scat = f32
    s = [None] * 6
    if split is not None:
        s = [split[k] for k in ("opac_L", "opac_R", "id", "chi_L", "chi_R", "chi_id")]
    use_flags = flags_in is not None
    o = NlRateOpts(int(split_rates), int(preconditioning), int(per_direction), int(use_flags),
                   int(scat is not None), 0, float(wmu), float(wtot))
    nwords = int(flags_in.shape[0]) if use_flags else 0
    lib().or_bb_rates(C.byref(st), C.byref(o), C.c_int(pop_ratio.size), _vp(b), _vp(nstar), _vp(pop_ratio),
                      _vp(e_kT), _vp(inv_df), _vp(vproj), _vp(adamp), _vp(tgx), _vp(th2x), _vp(work1), _vp(inu),
                      _vp(psi), _vp(irem), _vp(escape), _vp(beta), _vp(Bnu), *[_vp(a) for a in s], _vp(scat),
                      _vp(flags_in), _vp(flags_raise), C.c_int(nwords), _vp(gamma_ij), _vp(gamma_ji))


def bf_rates(win, b, nstar, e_kT, Jnu, PsiJ, beta, gamma_ij, gamma_ji, preconditioning=True):
    st, keep = make_window(win)
    b, nstar, e_kT = (_c(x, np.float64) for x in (b, nstar, e_kT))
    two = np.ascontiguousarray(win["twohnu3_c2"], np.float32)
    Jnu, PsiJ, beta = (_c(x, np.float32) for x in (Jnu, PsiJ, beta))
    lib().or_bf_rates(C.byref(st), C.c_int(e_kT.size), C.c_int(int(preconditioning)), _vp(b), _vp(nstar),
                      _vp(e_kT), _vp(two), _vp(Jnu), _vp(PsiJ), _vp(beta), _vp(gamma_ij), _vp(gamma_ji))


def normalize_profiles(atom, nstar, wphi, gamma_ij, gamma_ji, has_wphi, first_iter):
    ti = np.ascontiguousarray(atom["ti"], np.int32)
    tj = np.ascontiguousarray(atom["tj"], np.int32)
    act = None if atom.get("active") is None else np.ascontiguousarray(atom["active"], np.uint8)
    hw = np.ascontiguousarray(has_wphi, np.uint8)
    nstar = _c(nstar, np.float64)
    lib().or_normalize_profiles(C.c_int(gamma_ij.shape[1]), C.c_int(int(atom["nline"])), C.c_int(len(ti)), _vp(ti),
                                _vp(tj), _vp(act), _vp(hw), C.c_int(int(first_iter)), _vp(nstar), _vp(wphi),
                                _vp(gamma_ij), _vp(gamma_ji))


def lte_emission(chi, sigma, Bnu, beta, J=None, jmode=0, PsiJ=None, Jali=None, jali_valid=False, op_max=0.9):
    """Returns xhat, ehat, dJnu, n_negative; Jali updated in place."""
    chi, sigma, Bnu, beta, J, PsiJ = (_c(x, np.float32) for x in (chi, sigma, Bnu, beta, J, PsiJ))
    xhat, ehat, dj = np.empty_like(Bnu), np.empty_like(Bnu), np.empty_like(Bnu)
    f = lib().or_lte_emission
    f.restype = C.c_longlong
    neg = f(C.c_size_t(Bnu.size), _vp(chi), _vp(sigma), _vp(Bnu), _vp(beta), _vp(J), C.c_int(jmode), _vp(PsiJ),
            _vp(Jali), C.c_int(int(jali_valid)), C.c_double(op_max), _vp(xhat), _vp(ehat), _vp(dj))
    return xhat, ehat, dj, neg

"""ctypes front end of the statistical-equilibrium oracle (oracle/or_stateq.c).

TEST INFRASTRUCTURE ONLY: the checker of the SE kernels.  Atoms and per-cell
arrays have the layout of dispatch_b200.stateq (0-based indices, numpy arrays
(level or transition, cell) in C order, i.e. the cell index fastest).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import lib


class SqAtom(C.Structure):
    _fields_ = [("nlevel", C.c_int), ("nrad", C.c_int), ("nline", C.c_int), ("ncol", C.c_int),
                ("ti", C.c_void_p), ("tj", C.c_void_p), ("active", C.c_void_p), ("Aji", C.c_void_p),
                ("g", C.c_void_p), ("ev", C.c_void_p), ("ion", C.c_void_p),
                ("ci", C.c_void_p), ("cj", C.c_void_p), ("ckind", C.c_void_p), ("cfac", C.c_void_p),
                ("fmin", C.c_double), ("cbbesc", C.c_double), ("cbfesc", C.c_double), ("colscale", C.c_double),
                ("upsilon_floor", C.c_double), ("cut_x", C.c_double), ("bf_cut_rate", C.c_double),
                ("chkind", C.c_void_p), ("drawin", C.c_double), ("cbbhsc", C.c_double), ("cbfhsc", C.c_double),
                ("ngrec", C.c_int), ("ntemp", C.c_int), ("ch0_hmip", C.c_int), ("pad", C.c_int),
                ("gt", C.c_void_p), ("glnc", C.c_void_p), ("gdc", C.c_void_p),
                ("gll", C.c_void_p), ("gul", C.c_void_p), ("gkind", C.c_void_p), ("gcoll", C.c_void_p)]


class SqParams(C.Structure):
    _fields_ = [("max_update", C.c_double), ("sor_w", C.c_double), ("min_pop_frac", C.c_double),
                ("conv_pop_floor", C.c_double), ("tmax_update", C.c_double), ("cswitch", C.c_double),
                ("solver", C.c_int), ("pad", C.c_int)]


class SqResult(C.Structure):
    _fields_ = [("maxerr", C.c_double), ("epos_cell", C.c_longlong), ("epos_level", C.c_int), ("pad", C.c_int),
                ("nclamp", C.c_longlong), ("ntot", C.c_longlong), ("nonfinite_cell", C.c_longlong)]


def _vp(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def make_atom(atom: dict):
    keep = []

    def arr(key, dtype):
        v = atom.get(key)
        if v is None:
            return None
        a = np.ascontiguousarray(v, dtype)
        keep.append(a)
        return _vp(a)

    s = SqAtom()
    s.nlevel, s.nrad, s.nline = int(atom["nlevel"]), len(atom["ti"]), int(atom["nline"])
    s.ncol = len(atom["col_i"]) if atom.get("col_i") is not None else 0
    s.ti, s.tj, s.active, s.Aji = arr("ti", np.int32), arr("tj", np.int32), arr("active", np.uint8), arr("Aji", np.float64)
    s.g, s.ev, s.ion = arr("g", np.float64), arr("ev", np.float64), arr("ion", np.int32)
    s.ci, s.cj = arr("col_i", np.int32), arr("col_j", np.int32)
    s.ckind, s.cfac = arr("col_kind", np.int32), arr("col_fac", np.float32)
    for k, d in (("fmin", float(np.float32(1e-6))), ("cbbesc", 1.0), ("cbfesc", 1.0), ("colscale", 1.0),
                 ("upsilon_floor", 0.0), ("cut_x", 70.0), ("bf_cut_rate", 1.0)):
        setattr(s, k, float(atom.get(k, d)))
    s.chkind = arr("col_hkind", np.int32)
    s.drawin = prepare_drawin(float(atom["awgt"])) if s.chkind is not None else 0.0
    s.cbbhsc, s.cbfhsc = float(atom.get("cbbhsc", 1.0)), float(atom.get("cbfhsc", 1.0))
    gc = atom.get("gencol")
    if gc is not None and len(gc["ll"]) > 0:
        lnc = np.ascontiguousarray(gc["lnc"], np.float64)
        s.ngrec, s.ntemp = lnc.shape
        s.ch0_hmip = int(bool(gc.get("ch0_hmip", False)))
        tg = np.ascontiguousarray(gc["tgrid"], np.float64)
        dl = gc.get("dlnc")
        dl = hermite_derivative(tg, lnc) if dl is None else np.ascontiguousarray(dl, np.float64)
        keep.extend([lnc, tg, dl])
        s.gt, s.glnc, s.gdc = _vp(tg), _vp(lnc), _vp(dl)
        src = {"gll": gc["ll"], "gul": gc["ul"], "gkind": gc["kind"], "gcoll": gc.get("collider")}
        for k, v in src.items():
            if v is not None:
                a = np.ascontiguousarray(v, np.int32)
                keep.append(a)
                setattr(s, k, _vp(a))
    return s, keep


def hermite_derivative(tgrid, lnc):
    """hermite_derivative (pchip_slopes8) of every row of lnc (nrec, ntemp)."""
    tg = np.ascontiguousarray(tgrid, np.float64)
    lnc = np.ascontiguousarray(lnc, np.float64)
    out = np.zeros_like(lnc)
    for r in range(lnc.shape[0]):
        lib().sq_hermite_derivative(C.c_int(tg.size), _vp(tg), C.c_void_p(lnc[r].ctypes.data),
                                    C.c_void_p(out[r].ctypes.data))
    return out


def hermite_interp(x, y, d, xx):
    f = lib().sq_hermite_interp
    f.restype = C.c_double
    x, y, d = (np.ascontiguousarray(v, np.float64) for v in (x, y, d))
    return f(C.c_int(x.size), _vp(x), _vp(y), _vp(d), C.c_double(xx))


def collision_rows(atom: dict) -> int:
    ncol = len(atom["col_i"]) if atom.get("col_i") is not None else 0
    gc = atom.get("gencol")
    return ncol * (2 if atom.get("col_hkind") is not None else 1) + (2 * len(gc["ll"]) if gc is not None else 0)


def prepare_drawin(awgt: float) -> float:
    """prepare_Drawin (atom_mod.f90:1741-1750) for an atom of weight awgt [amu]."""
    f = lib().sq_prepare_drawin
    f.restype = C.c_double
    return f(C.c_double(awgt))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, np.float64)


def expin(x):
    f = lib().sq_expin
    f.restype = C.c_double
    return np.array([f(C.c_double(float(v))) for v in np.ravel(x)])


def kramer(lam, dev):
    f = lib().sq_kramer
    f.restype = C.c_double
    return f(C.c_double(lam), C.c_double(dev))


def collision_rates(atom: dict, temp, ne, e_kT, dxi=None, nh1=None, nstar=None, lsaha=None, colliders=None):
    """collision_rates' rows (collision_rows(atom), ncell): classic_col's upward
    electron rates, with col_hkind its hydrogen ones (reading nh1), then with
    gencol records their upward and downward rates (reading nstar, lsaha and,
    for UP/DN records, colliders (ncollider, ncell))."""
    st, keep = make_atom(atom)
    temp, ne, e_kT, dxi, nh1 = _f64(temp), _f64(ne), _f64(e_kT), _f64(dxi), _f64(nh1)
    nstar, lsaha, colliders = _f64(nstar), _f64(lsaha), _f64(colliders)
    if st.chkind is not None and nh1 is None:
        raise ValueError("hydrogen collision recipes need nh1")
    if st.ngrec > 0 and (nstar is None or lsaha is None):
        raise ValueError("gencol records need nstar and lsaha")
    cup = np.zeros((collision_rows(atom), temp.size), np.float64)
    lib().or_collisions(C.byref(st), C.c_int(temp.size), _vp(temp), _vp(ne), _vp(e_kT), _vp(dxi), _vp(nh1),
                        _vp(nstar), _vp(lsaha), _vp(colliders), _vp(cup))
    return cup


def solve(a, b, solver: int = 0):
    """One dense solve (0 lineq_no_pivot, 1 lineq, 2 LU partial pivot) of the
    column-major matrix a (numpy (n, n) is taken as a[i, j] = a(i, j))."""
    n = a.shape[0]
    af = np.asfortranarray(a, np.float64).copy(order="F")
    x = np.ascontiguousarray(b, np.float64).copy()
    fn = (lib().sq_lineq_no_pivot, lib().sq_lineq, lib().sq_lu_partial)[solver]
    fn(C.c_void_p(af.ctypes.data), _vp(x), C.c_int(n))
    return x


def rate_matrix(atom: dict, inputs: dict, cell: int, cup=None, cswitch: float = 1.0):
    """setup_transition_matrix of one cell: (W (n, n) with W[i, j] = w(i, j), e)."""
    st, keep = make_atom(atom)
    n = st.nlevel
    par = SqParams(100.0, 1.0, 1e-30, 0.0, 1e7, cswitch, 0, 0)
    bl = np.ascontiguousarray(inputs["b"][:, cell], np.float64)
    ns = np.ascontiguousarray(inputs["nstar"][:, cell], np.float64)
    gij = np.ascontiguousarray(inputs["gamma_ij"][:, cell], np.float32)
    gji = np.ascontiguousarray(inputs["gamma_ji"][:, cell], np.float32)
    cupc = (np.ascontiguousarray(cup[:, cell], np.float64) if cup is not None
            else np.zeros(max(collision_rows(atom), 1)))
    w = np.zeros(n * n, np.float64)
    e = np.zeros(n, np.float64)
    lib().or_rate_matrix(C.byref(st), C.byref(par), _vp(bl), _vp(ns), C.c_double(float(inputs["totn"][cell])),
                         C.c_double(float(inputs["e_kT"][cell])), _vp(gij), _vp(gji), _vp(cupc), _vp(w), _vp(e))
    return w.reshape(n, n).T.copy(), e


def stateq_update(atom: dict, b, nstar, totn, e_kT, gamma_ij, gamma_ji, temp=None, cup=None, solver: int = 0,
                  max_update: float = 1e2, sor_w: float = 1.0, min_pop_frac: float = 1e-30,
                  conv_pop_floor: float = 0.0, tmax_update: float = 1e7, cswitch: float = 1.0):
    """update_populations; b is updated in place; returns (result dict, lvlerr, status)."""
    st, keep = make_atom(atom)
    assert b.dtype == np.float64 and b.flags.c_contiguous
    nstar, totn, e_kT, temp, cup = _f64(nstar), _f64(totn), _f64(e_kT), _f64(temp), _f64(cup)
    gamma_ij = np.ascontiguousarray(gamma_ij, np.float32)
    gamma_ji = np.ascontiguousarray(gamma_ji, np.float32)
    if cswitch > 0 and (st.ncol > 0 or st.ngrec > 0) and cup is None:
        raise ValueError("the oracle takes the collision rates precomputed (collision_rates)")
    par = SqParams(max_update, sor_w, min_pop_frac, conv_pop_floor, tmax_update, cswitch, int(solver), 0)
    res = SqResult()
    lvlerr = np.zeros(st.nlevel, np.float64)
    rc = lib().or_stateq_update(C.byref(st), C.byref(par), C.c_int(totn.size), _vp(b), _vp(nstar), _vp(totn),
                                _vp(temp), _vp(e_kT), _vp(gamma_ij), _vp(gamma_ji), _vp(cup), C.byref(res),
                                _vp(lvlerr))
    out = {k: getattr(res, k) for k, _ in res._fields_ if k != "pad"}
    return out, lvlerr, rc


def ng_accumulate(b, oldb):
    b, oldb = _f64(b), _f64(oldb)
    gram = np.zeros(7)
    lib().or_ng_accumulate(C.c_int(b.shape[1]), C.c_int(b.shape[0]), _vp(b), _vp(oldb), _vp(gram))
    return gram


def ng_extrapolate(b, oldb, nstar, totn, a, bc, max_change=10.0):
    assert b.dtype == np.float64 and b.flags.c_contiguous
    oldb, nstar, totn = _f64(oldb), _f64(nstar), _f64(totn)
    emax, epc, epl = C.c_double(), C.c_longlong(), C.c_int()
    applied = lib().or_ng_extrapolate(C.c_int(b.shape[1]), C.c_int(b.shape[0]), _vp(b), _vp(oldb), _vp(nstar),
                                      _vp(totn), C.c_double(a), C.c_double(bc), C.c_double(max_change),
                                      C.byref(emax), C.byref(epc), C.byref(epl))
    return {"applied": bool(applied), "emax": emax.value, "epos_cell": epc.value, "epos_level": epl.value}

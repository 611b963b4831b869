"""ctypes front end of the sampled opacity table oracle (oracle/or_optab.c).

TEST INFRASTRUCTURE ONLY: the checker of the table kernels.  A table is a dict
lam (nnu,) fp64, val and optionally scat (nne, ntemp, nnu) fp32 (numpy order of
the Fortran (nnu, ntemp, nne)), pca a dict mu (2,), rot (2, 2) with rot[i, j] =
rot(i+1, j+1), c0 (2,), dc (2,).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import lib


class Pca(C.Structure):
    _fields_ = [("mu", C.c_double * 2), ("rot", C.c_double * 4), ("c0", C.c_double * 2), ("dc", C.c_double * 2)]


def make_pca(pca: dict) -> Pca:
    r = np.asarray(pca["rot"], np.float64)
    return Pca((C.c_double * 2)(*pca["mu"]), (C.c_double * 4)(r[0, 0], r[1, 0], r[0, 1], r[1, 1]),
               (C.c_double * 2)(*pca["c0"]), (C.c_double * 2)(*pca["dc"]))


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _shape(tab):
    nne, ntemp, nnu = np.shape(tab["val"])
    return nnu, ntemp, nne


def slopes(tab: dict, component: str = "val"):
    """sample_build_derivatives (optab_mod.f90:125-166): (dl, dt, de) of one component."""
    nnu, ntemp, nne = _shape(tab)
    lam = np.ascontiguousarray(tab["lam"], np.float64)
    v = np.ascontiguousarray(tab[component], np.float32)
    out = [np.zeros_like(v) for _ in range(3)]
    lib().or_optab_slopes(C.c_int(nnu), C.c_int(ntemp), C.c_int(nne), _p(lam), _p(v), C.byref(make_pca(tab["pca"])),
                          *[_p(o) for o in out])
    return tuple(out)


def _all_slopes(tab):
    s = slopes(tab, "val")
    t = slopes(tab, "scat") if tab.get("scat") is not None else (None, None, None)
    return s, t


def sample(tab: dict, temp, ne, chi500, lam_q):
    """sample_interpolate (optab_mod.f90:181-287): (back, scat), each (ncell, nf)."""
    nnu, ntemp, nne = _shape(tab)
    (dl, dt, de), (sl, st, se) = _all_slopes(tab)
    T, N = np.ascontiguousarray(temp, np.float64).ravel(), np.ascontiguousarray(ne, np.float64).ravel()
    ch = np.ascontiguousarray(chi500, np.float32).ravel()
    q = np.ascontiguousarray(lam_q, np.float64)
    back = np.zeros((T.size, q.size), np.float32)
    scat = np.zeros_like(back)
    val = np.ascontiguousarray(tab["val"], np.float32)
    sv = np.ascontiguousarray(tab["scat"], np.float32)
    lam = np.ascontiguousarray(tab["lam"], np.float64)
    f = lib().or_optab_sample
    f.argtypes = [C.c_int] * 3 + [C.c_void_p] * 10 + [C.c_longlong] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3
    rc = f(nnu, ntemp, nne, _p(lam), C.byref(make_pca(tab["pca"])), _p(val), _p(dl), _p(dt), _p(de), _p(sv), _p(sl),
           _p(st), _p(se), T.size, _p(T), _p(N), _p(ch), q.size, _p(q), _p(back), _p(scat))
    if rc:
        raise RuntimeError(f"oracle optab_sample rc={rc}")
    return back, scat


def sample_ll(tab: dict, temp, ne, chi500, vproj, lam_q, xhat, ehat, chi_scat=None):
    """sample_interpolate_ll (optab_mod.f90:300-409) in place on xhat, ehat and
    chi_scat (ncell, nf) fp32."""
    nnu, ntemp, nne = _shape(tab)
    (dl, dt, de), (sl, st, se) = _all_slopes(tab)
    T, N = np.ascontiguousarray(temp, np.float64).ravel(), np.ascontiguousarray(ne, np.float64).ravel()
    ch = np.ascontiguousarray(chi500, np.float32).ravel()
    vp = np.ascontiguousarray(vproj, np.float32).ravel()
    q = np.ascontiguousarray(lam_q, np.float64)
    for a in (xhat, ehat, chi_scat):
        assert a is None or (a.dtype == np.float32 and a.flags.c_contiguous and a.size == T.size * q.size)
    val = np.ascontiguousarray(tab["val"], np.float32)
    sv = None if tab.get("scat") is None else np.ascontiguousarray(tab["scat"], np.float32)
    lam = np.ascontiguousarray(tab["lam"], np.float64)
    f = lib().or_optab_sample_ll
    f.argtypes = ([C.c_int] * 3 + [C.c_void_p] * 10 + [C.c_longlong] + [C.c_void_p] * 4 + [C.c_int]
                  + [C.c_void_p] * 4)
    rc = f(nnu, ntemp, nne, _p(lam), C.byref(make_pca(tab["pca"])), _p(val), _p(dl), _p(dt), _p(de), _p(sv), _p(sl),
           _p(st), _p(se), T.size, _p(T), _p(N), _p(ch), _p(vp), q.size, _p(q), _p(xhat), _p(ehat), _p(chi_scat))
    if rc:
        raise RuntimeError(f"oracle optab_sample_ll rc={rc}")

"""ctypes front end of the continuum-opacity oracle (oracle/or_continuum.c).

TEST INFRASTRUCTURE ONLY: the checker of the continuum kernels.  Components and
cells are the dicts of dispatch_b200.continuum; the structs are declared here
again (their layout is the C header's), so the checker does not share the
product's packing code.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import lib

_FLAGS = ("ilogl", "kvadl", "minex", "maxex", "loglam", "kvadt", "minet", "maxet", "iteta", "lam3", "log_table")
_CELL = ("n", "n2", "part", "level_n", "level_w")


class _Comp(C.Structure):
    _fields_ = ([("kind", C.c_int), ("istim", C.c_int), ("nnu", C.c_int), ("ntt", C.c_int)]
                + [(k, C.c_int) for k in _FLAGS] + [("k", C.c_int)]
                + [(k, C.c_void_p) for k in ("lam", "lnlam", "tt", "xkap", "ldisk")]
                + [(k, C.c_double) for k in ("xkap_scale", "mint", "maxt", "minl", "maxl", "ion_xion", "level_g",
                                             "level_xion", "awgt")]
                + [(k, C.c_void_p) for k in _CELL[:4]]
                + [(k, C.c_int) for k in ("occupation", "dissolved_only", "level_i", "pad2")]
                + [("level_w", C.c_void_p)])


class _Cells(C.Structure):
    _fields_ = ([(k, C.c_void_p) for k in ("temp", "teta", "e_kT", "pe", "dxi", "ne", "nHI", "partHI", "nHeI",
                                           "nH2")]
                + [("HI_xion", C.c_double), ("helium_scattering", C.c_int), ("pad", C.c_int),
                   ("shield", C.c_void_p)])


def _pack(comps, keep):
    arr = (_Comp * max(len(comps), 1))()
    for s, c in zip(arr, comps):
        lam = np.ascontiguousarray(c["lam"], np.float64)
        tt = np.ascontiguousarray(c["tt"], np.float64)
        xk = np.ascontiguousarray(c["xkap"], np.float32)
        ld = np.ascontiguousarray(c.get("ldisk", np.zeros(lam.size, bool)), np.uint8)
        lnlam = np.log(lam)
        keep += [lam, tt, xk, ld, lnlam]
        s.kind, s.istim, s.nnu, s.ntt, s.k = int(c["kind"]), int(c.get("istim", 0)), lam.size, tt.size, int(c.get("k", 0))
        for k in _FLAGS:
            setattr(s, k, int(bool(c.get(k, False))))
        s.lam, s.lnlam, s.tt, s.xkap, s.ldisk = (a.ctypes.data for a in (lam, lnlam, tt, xk, ld))
        for k in ("xkap_scale", "mint", "maxt", "minl", "maxl", "ion_xion", "level_g", "level_xion", "awgt"):
            setattr(s, k, float(c.get(k, 0.0)))
        s.occupation, s.dissolved_only = int(bool(c.get("occupation", False))), int(bool(c.get("dissolved_only", False)))
        s.level_i = int(c.get("level_i", 0))
        for k in _CELL:
            a = c.get(k)
            if a is not None:
                a = np.ascontiguousarray(a, np.float64)
                keep.append(a)
                setattr(s, k, a.ctypes.data)
    return arr


def bf_weights(comp: dict, lam):
    """load_lam_interp_weights of one component: (active, iw (0-based, -1 none),
    quad, lagrange (nlam, 3), fs, fe)."""
    keep = []
    arr = _pack([comp], keep)
    lam = np.ascontiguousarray(lam, np.float64)
    n = lam.size
    iw = np.empty(n, np.int32)
    quad = np.empty(n, np.uint8)
    lag = np.empty((n, 3), np.float32)
    fs, fe = C.c_int(), C.c_int()
    f = lib().or_bf_weights
    f.restype = C.c_int
    act = f(C.byref(arr[0]), C.c_int(n), C.c_void_p(lam.ctypes.data), C.c_void_p(iw.ctypes.data),
            C.c_void_p(quad.ctypes.data), C.c_void_p(lag.ctypes.data), C.byref(fs), C.byref(fe))
    return bool(act), iw, quad.astype(bool), lag, fs.value, fe.value


def continuum_opacities(comps: list, lam, nu, cells: dict, beta=None, sigma: bool = True):
    """(xhat, sigma or None), each (ncell, nlam) float32."""
    keep = []
    arr = _pack(comps, keep)
    s = _Cells()
    for k in ("temp", "teta", "e_kT", "pe", "dxi", "ne", "nHI", "partHI", "nHeI", "nH2", "shield"):
        a = cells.get(k)
        if a is not None:
            a = np.ascontiguousarray(a, np.float64)
            keep.append(a)
            setattr(s, k, a.ctypes.data)
    s.HI_xion = float(cells.get("HI_xion", 13.598434))
    s.helium_scattering = int(bool(cells.get("helium_scattering", True)))
    lam = np.ascontiguousarray(lam, np.float64)
    nu = None if nu is None else np.ascontiguousarray(nu, np.float64)
    ncell, nlam = int(np.asarray(cells["temp"]).shape[0]), lam.size
    xhat = np.empty((ncell, nlam), np.float32)
    sg = np.empty_like(xhat) if sigma else None
    beta = None if beta is None else np.ascontiguousarray(beta, np.float32)
    f = lib().or_continuum_opacities
    f.restype = C.c_int
    rc = f(C.c_int(len(comps)), arr, C.c_int(nlam), C.c_void_p(lam.ctypes.data),
           None if nu is None else C.c_void_p(nu.ctypes.data), C.c_int(ncell), C.byref(s),
           None if beta is None else C.c_void_p(beta.ctypes.data), C.c_void_p(xhat.ctypes.data),
           None if sg is None else C.c_void_p(sg.ctypes.data))
    if rc != 0:
        raise ValueError("or_continuum_opacities: unsupported component")
    return xhat, sg


def h_levels(cells: dict, nk: int, occupation: bool = True):
    """init_H_levels with compute_shield: (shield (ncell,), level_n (nk, ncell),
    level_w (nk, ncell) or None)."""
    arr = {k: (None if cells.get(k) is None else np.ascontiguousarray(cells[k], np.float64))
           for k in ("temp", "e_kT", "ne", "dxi", "nHI", "nHeI", "partHI")}
    n = arr["temp"].size
    sh = np.empty(n)
    ln = np.empty((nk, n))
    lw = np.empty((nk, n)) if occupation else None
    p = lambda a: None if a is None else C.c_void_p(a.ctypes.data)
    lib().or_h_levels(C.c_int(n), C.c_int(nk), C.c_int(int(occupation)), p(arr["temp"]), p(arr["e_kT"]),
                      p(arr["ne"]), p(arr["dxi"]), p(arr["nHI"]), p(arr["nHeI"]), p(arr["partHI"]), p(sh), p(ln), p(lw))
    return sh, ln, lw

"""The continuum opacity of a frequency window on the device: HOP's
composition_type%continuum_opacities (HOP/composition_mod.f90:2893-2984) through
m3d_continuum_opacities.

A component is a dict holding an absdat component's table and flags (bftrans_type,
HOP/bftrans_mod.f90:19-52) and the number densities its absorption factor reads;
the cells dict holds the EOS state.  An 'H BF' level under occupation
probabilities (the reference's default H_occupation_probability) sets
occupation=True, level_i (principal quantum number), level_xion (its excitation
energy [eV]), level_n and level_w (its population and occupation probability per
cell), n (H I's density), and optionally dissolved_only; its cells need ne, nHeI and
shield ((1+a)^3.15/ne of composition_type%compute_shield).  Cell arrays are numpy (host) or CUDA tensors
(device, then the outputs are CUDA tensors too); tables are numpy.

    xhat, sigma = continuum_opacities(comps, lam, nu, cells)

xhat and sigma are (ncell, nlam): the working-form true absorption and the
electron + Rayleigh scattering opacity [1/cm].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DEVICE_PTRS, M3DError, check, init, lib, order_after_torch, ptr

# absorption_factor's cases (bftrans_mod.f90:500-528), M3D_BF_* of the C header
HMINUS, NPE, H, H_FF, PAIR, H2PLUS, PEDEP, PEACH, MOLECULAR, REGULAR = range(1, 11)

_FLAGS = ("ilogl", "kvadl", "minex", "maxex", "loglam", "kvadt", "minet", "maxet", "iteta", "lam3", "log_table")
_CELL = ("n", "n2", "part", "level_n", "level_w")


class BfComp(C.Structure):
    """m3d_bf_comp_t."""

    _fields_ = ([("kind", C.c_int), ("istim", C.c_int), ("nnu", C.c_int), ("ntt", C.c_int)]
                + [(k, C.c_int) for k in _FLAGS] + [("k", C.c_int)]
                + [("lam", C.c_void_p), ("lnlam", C.c_void_p), ("tt", C.c_void_p), ("xkap", C.c_void_p),
                   ("ldisk", C.c_void_p)]
                + [(k, C.c_double) for k in ("xkap_scale", "mint", "maxt", "minl", "maxl", "ion_xion", "level_g",
                                             "level_xion", "awgt")]
                + [(k, C.c_void_p) for k in _CELL[:4]]
                + [(k, C.c_int) for k in ("occupation", "dissolved_only", "level_i", "pad2")]
                + [("level_w", C.c_void_p)])


class ContCells(C.Structure):
    """m3d_cont_cells_t."""

    _fields_ = ([(k, C.c_void_p) for k in ("temp", "teta", "e_kT", "pe", "dxi", "ne", "nHI", "partHI", "nHeI",
                                           "nH2")]
                + [("HI_xion", C.c_double), ("helium_scattering", C.c_int), ("pad", C.c_int),
                   ("shield", C.c_void_p)])


def set_table(xkap, ilogt: bool, ilogl: bool):
    """bftrans_type%set_table (bftrans_mod.f90:77-91): the stored form of a table
    xkap (ntt, nnu) as read -- divided by its maximum, logarithmic for a logarithmic
    temperature interpolation (or, without temperature dependence, a logarithmic
    wavelength one), ln of 1e-37 for non-positive entries.  Returns (xkap float32
    (ntt, nnu), xkap_scale, log_table)."""
    xkap = np.asarray(xkap, np.float64)
    ntt = xkap.shape[0]
    log_table = bool(ilogt if ntt > 1 else ilogl)
    scale = float(xkap.max())
    if scale <= 0:
        scale = 1.0
    if log_table:
        stored = (np.log(np.where(xkap > 0, xkap, 1e-37)) - np.log(scale)).astype(np.float32)
    else:
        stored = (xkap / scale).astype(np.float32)
    return np.ascontiguousarray(stored), scale, log_table


def _cell_array(a, dev: bool):
    if a is None:
        return None
    if dev:
        return a.contiguous()
    return np.ascontiguousarray(a, np.float64)


def make_comps(comps: list, dev: bool = False):
    """(array of BfComp, the arrays it points into)."""
    n = len(comps)
    arr = (BfComp * max(n, 1))()
    keep = []
    for s, c in zip(arr, comps):
        lam = np.ascontiguousarray(c["lam"], np.float64)
        tt = np.ascontiguousarray(c["tt"], np.float64)
        xk = np.ascontiguousarray(c["xkap"], np.float32)
        ld = np.ascontiguousarray(c.get("ldisk", np.zeros(lam.size, bool)), np.uint8)
        lnlam = np.log(lam)
        keep += [lam, tt, xk, ld, lnlam]
        s.kind, s.istim, s.nnu, s.ntt = int(c["kind"]), int(c.get("istim", 0)), lam.size, tt.size
        if xk.shape != (tt.size, lam.size):
            raise M3DError(f"continuum: xkap must be (ntt, nnu) = ({tt.size}, {lam.size}), got {xk.shape}")
        for k in _FLAGS:
            setattr(s, k, int(bool(c.get(k, False))))
        s.k = int(c.get("k", 0))
        s.lam, s.lnlam, s.tt, s.xkap, s.ldisk = (a.ctypes.data for a in (lam, lnlam, tt, xk, ld))
        for k in ("xkap_scale", "mint", "maxt", "minl", "maxl", "ion_xion", "level_g", "level_xion", "awgt"):
            setattr(s, k, float(c.get(k, 0.0)))
        s.occupation, s.dissolved_only = int(bool(c.get("occupation", False))), int(bool(c.get("dissolved_only", False)))
        s.level_i = int(c.get("level_i", 0))
        for k in _CELL:
            a = _cell_array(c.get(k), dev)
            keep.append(a)
            setattr(s, k, ptr(a).value if a is not None else None)
    return arr, keep


def make_cells(cells: dict, dev: bool = False):
    s = ContCells()
    keep = []
    for k in ("temp", "teta", "e_kT", "pe", "dxi", "ne", "nHI", "partHI", "nHeI", "nH2", "shield"):
        a = _cell_array(cells.get(k), dev)
        keep.append(a)
        setattr(s, k, ptr(a).value if a is not None else None)
    s.HI_xion = float(cells.get("HI_xion", 13.598434))
    s.helium_scattering = int(bool(cells.get("helium_scattering", True)))
    return s, keep


def continuum_opacities(comps: list, lam, nu, cells: dict, beta=None, sigma: bool = True):
    """(xhat, sigma or None), each (ncell, nlam): numpy for host cells, CUDA tensors
    for device cells (the cells dict's arrays all on one side)."""
    init()
    dev = not isinstance(cells["temp"], np.ndarray)
    lam = np.ascontiguousarray(lam, np.float64)
    nu = None if nu is None else np.ascontiguousarray(nu, np.float64)
    ncell, nlam = int(cells["temp"].shape[0]), int(lam.size)
    arr, keep = make_comps(comps, dev)
    cs, keep2 = make_cells(cells, dev)
    if dev:
        import torch
        xhat = torch.empty((ncell, nlam), dtype=torch.float32, device=cells["temp"].device)
        sg = torch.empty_like(xhat) if sigma else None
        beta = None if beta is None else beta.contiguous()
        order_after_torch(cells["temp"])
        flags = DEVICE_PTRS
    else:
        xhat = np.empty((ncell, nlam), np.float32)
        sg = np.empty_like(xhat) if sigma else None
        beta = None if beta is None else np.ascontiguousarray(beta, np.float32)
        flags = 0
    check(lib().m3d_continuum_opacities(C.c_int(len(comps)), arr, C.c_int(nlam), C.c_void_p(lam.ctypes.data),
                                        None if nu is None else C.c_void_p(nu.ctypes.data), C.c_int(ncell),
                                        C.byref(cs), ptr(beta), ptr(xhat), ptr(sg), C.c_uint(flags)),
          "m3d_continuum_opacities")
    del keep, keep2
    return xhat, sg


def opacity(comps: list, lam, nu, cells: dict, beta=None, include_llist: bool = True, line_margin: float = 100.0,
            disjoint: bool = False):
    """composition_type%opacity (HOP/composition_mod.f90:3122-3260) through
    m3d_opacity: the continuum of comps and cells, the line list of the state loaded
    with hop_set_state (same cells) against it, and the conversion to physical
    extinction.  Returns (chi, scat), each (ncell, nlam) float32: chi the total
    extinction (the true absorption alone with disjoint), scat electron + Rayleigh
    scattering.  Host arrays."""
    init()
    lam = np.ascontiguousarray(lam, np.float64)
    nu = np.ascontiguousarray(nu, np.float64)
    ncell, nlam = int(np.asarray(cells["temp"]).shape[0]), int(lam.size)
    arr, keep = make_comps(comps, False)
    cs, keep2 = make_cells(cells, False)
    chi = np.empty((ncell, nlam), np.float32)
    scat = np.empty_like(chi)
    beta = None if beta is None else np.ascontiguousarray(beta, np.float32)
    check(lib().m3d_opacity(C.c_int(nlam), C.c_void_p(lam.ctypes.data), C.c_void_p(nu.ctypes.data), C.c_int(ncell),
                            C.c_int(len(comps)), arr, C.byref(cs), ptr(beta), ptr(chi), ptr(scat),
                            C.c_int(int(bool(include_llist))), C.c_double(line_margin), C.c_int(int(bool(disjoint)))),
          "m3d_opacity")
    del keep, keep2
    return chi, scat


def h_levels(cells: dict, nk: int, occupation: bool = True):
    """The H I level set-up the 'H BF' components read (init_H_levels with
    compute_shield, HOP/composition_mod.f90:2604-2613, 2708-2768) through m3d_h_levels:
    (shield (ncell,), level_n (nk, ncell), level_w (nk, ncell) or None), numpy for host
    cells, CUDA tensors for device cells.  cells needs temp, e_kT, ne, dxi, nHI, and
    nHeI (with occupation) or partHI (without)."""
    init()
    dev = not isinstance(cells["temp"], np.ndarray)
    arr = {k: _cell_array(cells.get(k), dev) for k in ("temp", "e_kT", "ne", "dxi", "nHI", "nHeI", "partHI")}
    n = int(cells["temp"].shape[0])
    if dev:
        import torch
        dv = cells["temp"].device
        sh = torch.empty(n, dtype=torch.float64, device=dv)
        ln = torch.empty((nk, n), dtype=torch.float64, device=dv)
        lw = torch.empty((nk, n), dtype=torch.float64, device=dv) if occupation else None
        order_after_torch(cells["temp"])
        flags = DEVICE_PTRS
    else:
        sh, ln = np.empty(n), np.empty((nk, n))
        lw = np.empty((nk, n)) if occupation else None
        flags = 0
    check(lib().m3d_h_levels(C.c_int(n), C.c_int(nk), C.c_int(int(occupation)),
                             *[ptr(arr[k]) for k in ("temp", "e_kT", "ne", "dxi", "nHI", "nHeI", "partHI")],
                             ptr(sh), ptr(ln), ptr(lw), C.c_uint(flags)), "m3d_h_levels")
    return sh, ln, lw


def airvac_corr(lam):
    """The refractive index of air at wavelength lam [AA] (HOP/handyfuncs_mod.f90:437-445),
    the published formula VALD uses (Piskunov, after Ciddor 1996)."""
    s2 = (1e4 / np.asarray(lam, np.float64)) ** 2
    return 1.00008336624212083 + 0.02408926869968 / (130.1065924522 - s2) + 0.0001599740894897 / (38.92568793293 - s2)


def air2vac(air):
    """Vacuum wavelength [AA] of the air wavelength air [AA]: the index evaluated at the
    vacuum wavelength by three substitutions (HOP/handyfuncs_mod.f90:424-431)."""
    air = np.asarray(air, np.float64)
    w = air * airvac_corr(air)
    w = air * airvac_corr(w)
    return air * airvac_corr(w)


def chi500(comps: list, cells: dict, ref_lam: float = 5000.0):
    """load_state_variables' reference opacity (HOP/composition_mod.f90:2169-2176): the
    total extinction at the vacuum wavelength of ref_lam [AA] air, continuum and
    scattering without the line list (ncell,), float32."""
    lam = np.atleast_1d(air2vac(ref_lam))
    nu = (2.99792458e10 / 1e-8) / lam       # HZ_TO_AA / lambda (const_mod.f90:57)
    chi, _ = opacity(comps, lam, nu, cells, include_llist=False)
    return chi[:, 0]


__all__ = ["continuum_opacities", "opacity", "chi500", "air2vac", "h_levels", "set_table", "BfComp", "ContCells", "HMINUS", "NPE", "H", "H_FF", "PAIR",
           "H2PLUS", "PEDEP", "PEACH", "MOLECULAR", "REGULAR"]

"""ctypes front end of the hydrogen line-profile oracle (oracle/or_hprof.c).

TEST INFRASTRUCTURE ONLY: the checker of the hydrogen kernels.  Cell fields are
flat numpy arrays; chi, eta and cont are (ncell, nf) float32.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .oracle import lib, qlg_tables

CELL_FIELDS = ("vproj", "inv_df", "temp", "ni", "ne", "tothi", "vbar2h", "fo", "t3nhe")


class HLine(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("bpo", C.c_int), ("io", C.c_int), ("opts", C.c_int),
                ("pad", C.c_int), ("nu0", C.c_double),
                ("grad", C.c_double), ("gstk", C.c_double), ("gw1", C.c_double), ("gw2", C.c_double),
                ("gw3", C.c_double), ("dq", C.c_double * 14), ("wt", C.c_double * 14), ("dqbar", C.c_double),
                ("dqmax", C.c_double), ("qray", C.c_double)]


class HCells(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in CELL_FIELDS]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def hydrogen_line(n, m, nu0, opts=0) -> HLine:
    h = HLine()
    lib().or_hydrogen_line(C.c_int(n), C.c_int(m), C.c_double(nu0), C.c_uint(opts), C.byref(h))
    return h


def hprofile(h: HLine, cell: dict, q):
    """hcell_prepare + hprofile in one cell at the detunings q."""
    tgx, th2x = qlg_tables()
    q = np.ascontiguousarray(q, np.float64)
    phi = np.zeros(q.size, np.float32)
    f = lib().or_hprofile
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_float] * 7 + [C.c_int, C.c_void_p, C.c_void_p]
    f(C.byref(h), _p(tgx), _p(th2x), *[float(cell[k]) for k in ("temp", "ne", "fo", "vbar2h", "tothi", "t3nhe",
                                                                "inv_df")], q.size, _p(q), _p(phi))
    return phi


def add_h_opacities(h: HLine, Bij, f0, nu, cells: dict, chi, eta, cont, bi=None, bj=None):
    """add_h_opacities in place on chi, eta (ncell, nf); returns (line_used, line_strength)."""
    tgx, th2x = qlg_tables()
    keep = {k: np.ascontiguousarray(cells[k], np.float32).ravel() for k in CELL_FIELDS}
    hc = HCells(*[keep[k].ctypes.data for k in CELL_FIELDS])
    nu = np.ascontiguousarray(nu, np.float64)
    bi = None if bi is None else np.ascontiguousarray(bi, np.float32)
    bj = None if bj is None else np.ascontiguousarray(bj, np.float32)
    for a in (chi, eta):
        assert a.dtype == np.float32 and a.flags.c_contiguous
    cont = np.ascontiguousarray(cont, np.float32)
    used = C.c_int(0)
    strength = C.c_float(0.0)
    f = lib().or_add_h_opacities
    f.argtypes = [C.c_void_p] * 3 + [C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_longlong] + [C.c_void_p] * 8
    f(C.byref(h), _p(tgx), _p(th2x), float(Bij), int(f0), nu.size, _p(nu), keep["temp"].size, C.byref(hc),
      _p(bi), _p(bj), _p(chi), _p(eta), _p(cont), C.byref(used), C.byref(strength))
    return bool(used.value), float(strength.value)


def vcs_load(series: int, path: str, radiative: bool) -> None:
    """read_vcs_grid of one series (1 Balmer, 2 Paschen, 3 Brackett)."""
    rc = lib().or_vcs_load(C.c_int(series), str(path).encode(), C.c_int(int(radiative)))
    if rc:
        raise RuntimeError(f"oracle vcs_load({series}, {path}) rc={rc}")


def vcs_clear() -> None:
    lib().or_vcs_clear()

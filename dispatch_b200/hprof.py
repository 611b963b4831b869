"""Hydrogen line profiles (HOP/hprofl_mod.f90, the analytic path) on the device.

hydrogen_line(n, m, nu0) returns the line's constants (hline_t) from the host;
profile() evaluates hcell_prepare + hprofile per cell at given detunings, and
add_h_opacities() adds one line to chi and eta as the reference's walk does.
Arrays are numpy (host buffers) or torch CUDA tensors (device pointers); cell
fields flat (ncell,), (frequency, cell) arrays in numpy order (ncell, nf).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DEVICE_PTRS, check, init, lib, ptr
from .rt import _is_dev

CELL_FIELDS = ("vproj", "inv_df", "temp", "ni", "ne", "tothi", "vbar2h", "fo", "t3nhe")
NO_RAD, NO_STARK, NO_VDW, NO_BPO = 1, 2, 4, 8


class HLine(C.Structure):
    """m3d_hline_t."""

    _fields_ = [("n", C.c_int), ("m", C.c_int), ("bpo", C.c_int), ("io", C.c_int), ("opts", C.c_int),
                ("pad", C.c_int), ("nu0", C.c_double),
                ("grad", C.c_double), ("gstk", C.c_double), ("gw1", C.c_double), ("gw2", C.c_double),
                ("gw3", C.c_double), ("dq", C.c_double * 14), ("wt", C.c_double * 14), ("dqbar", C.c_double),
                ("dqmax", C.c_double), ("qray", C.c_double)]


class HCells(C.Structure):
    """m3d_hcells_t."""

    _fields_ = [(k, C.c_void_p) for k in CELL_FIELDS]


def hydrogen_line(n: int, m: int, nu0: float, opts: int = 0) -> HLine:
    """hydrogen_line (hprofl_mod.f90:703-810), computed on the host (no device needed)."""
    h = HLine()
    check(lib().m3d_hydrogen_line(C.c_int(n), C.c_int(m), C.c_double(nu0), C.c_uint(opts), C.byref(h)),
          "m3d_hydrogen_line")
    return h


def _cells(cells: dict, dev: bool):
    keep = [cells[k] if dev else np.ascontiguousarray(cells[k], np.float32).ravel() for k in CELL_FIELDS]
    return HCells(*[ptr(a).value if ptr(a) is not None else None for a in keep]), keep


def profile(h: HLine, cells: dict, q):
    """phi (ncell, nq) of the line in each cell at the detunings q."""
    init()
    dev = _is_dev(cells["temp"])
    hc, keep = _cells(cells, dev)
    ncell = int(np.prod(cells["temp"].shape))
    if dev:
        import torch
        qd = q if not isinstance(q, np.ndarray) else torch.from_numpy(np.ascontiguousarray(q, np.float64)).cuda()
        phi = torch.empty((ncell, qd.numel()), dtype=torch.float32, device="cuda")
    else:
        qd = np.ascontiguousarray(q, np.float64)
        phi = np.empty((ncell, qd.size), np.float32)
    nq = int(qd.shape[0])
    check(lib().m3d_h_profile(C.byref(h), C.c_longlong(ncell), C.byref(hc), C.c_int(nq), ptr(qd), ptr(phi),
                              C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_h_profile")
    del keep
    return phi


def add_h_opacities(h: HLine, Bij: float, f0: int, nu, cells: dict, chi, eta, cont, bi=None, bj=None):
    """add_h_opacities in place on chi, eta; returns (line_used, line_strength)."""
    init()
    dev = _is_dev(chi)
    hc, keep = _cells(cells, dev)
    conv = (lambda a, dt: a) if dev else (lambda a, dt: None if a is None else np.ascontiguousarray(a, dt))
    nu_, cont_, bi_, bj_ = conv(nu, np.float64), conv(cont, np.float32), conv(bi, np.float32), conv(bj, np.float32)
    used = C.c_int(0)
    strength = C.c_float(0.0)
    nf = int(nu_.shape[0])
    ncell = int(np.prod(cells["temp"].shape))
    check(lib().m3d_h_opacity(C.byref(h), C.c_double(Bij), C.c_int(f0), C.c_int(nf), ptr(nu_), C.c_longlong(ncell),
                              C.byref(hc), ptr(bi_), ptr(bj_), ptr(chi), ptr(eta), ptr(cont_), C.byref(used),
                              C.byref(strength), C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_h_opacity")
    del keep
    return bool(used.value), float(strength.value)


def vcs_load(series: int, path: str, radiative: bool) -> None:
    """read_vcs_grid of one series (1 Balmer, 2 Paschen, 3 Brackett)."""
    init()
    check(lib().m3d_vcs_load(C.c_int(series), str(path).encode(), C.c_int(int(radiative))), "m3d_vcs_load")


def vcs_clear() -> None:
    init()
    lib().m3d_vcs_clear()


def vcs_supported(n: int, m: int) -> bool:
    return bool(lib().m3d_vcs_supported(C.c_int(n), C.c_int(m)))

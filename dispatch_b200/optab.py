"""The sampled opacity tables of HOP/optab_mod.f90 on the device.

SampleOptab mirrors sample_optab_type (optab_mod.f90:37-77): it is built from
the wavelength nodes, the value and scattering components and the PCA transform
of (ln T, ln ne), computes its node slopes at construction (build_derivatives,
:125-166) and stays resident on the device; interpolate (:181-287) and
interpolate_ll (:300-409) sample it per (frequency, cell).  Arrays are numpy
(host buffers) or torch CUDA tensors (device pointers); tables and (f, cell)
arrays in numpy order, i.e. (nne, ntemp, nnu) and (ncell, nf).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DEVICE_PTRS, check, init, lib, ptr
from .rt import _is_dev


class Pca(C.Structure):
    """m3d_pca_t."""

    _fields_ = [("mu", C.c_double * 2), ("rot", C.c_double * 4), ("c0", C.c_double * 2), ("dc", C.c_double * 2)]


def make_pca(pca: dict) -> Pca:
    """pca: mu (2,), rot (2, 2) with rot[i, j] = rot(i+1, j+1), c0 (2,), dc (2,)."""
    r = np.asarray(pca["rot"], np.float64)
    return Pca((C.c_double * 2)(*pca["mu"]), (C.c_double * 4)(r[0, 0], r[1, 0], r[0, 1], r[1, 1]),
               (C.c_double * 2)(*pca["c0"]), (C.c_double * 2)(*pca["dc"]))


class SampleOptab:
    """A sampled opacity table resident on the device (m3d_optab_t)."""

    def __init__(self, lam, val, scat, pca: dict):
        init()
        dev = _is_dev(val)
        self.nne, self.ntemp, self.nnu = (int(n) for n in val.shape)
        conv = (lambda a, dt: a) if dev else (lambda a, dt: None if a is None else np.ascontiguousarray(a, dt))
        keep = [conv(lam, np.float64), conv(val, np.float32), conv(scat, np.float32)]
        self.has_scat = scat is not None
        h = C.c_void_p()
        check(lib().m3d_optab_create(C.c_int(self.nnu), C.c_int(self.ntemp), C.c_int(self.nne), ptr(keep[0]),
                                     ptr(keep[1]), ptr(keep[2]), C.byref(make_pca(pca)),
                                     C.c_uint(DEVICE_PTRS if dev else 0), C.byref(h)), "m3d_optab_create")
        self._h = h

    @classmethod
    def from_dict(cls, tab: dict) -> "SampleOptab":
        return cls(tab["lam"], tab["val"], tab.get("scat"), tab["pca"])

    def slopes(self, component: int = 0):
        """(dl, dt, de) node slopes of the value (0) or scattering (1) component."""
        out = [np.empty((self.nne, self.ntemp, self.nnu), np.float32) for _ in range(3)]
        check(lib().m3d_optab_slopes(self._h, C.c_int(component), *[ptr(o) for o in out], C.c_uint(0)),
              "m3d_optab_slopes")
        return tuple(out)

    def interpolate(self, temp, ne, chi500, lam_q, back=None, scat=None):
        """sample_interpolate: returns (back, scat), (ncell, nf)."""
        dev = _is_dev(temp, ne, chi500, lam_q)
        ncell, nf = int(np.prod(temp.shape)), int(lam_q.shape[0])
        if back is None:
            back, scat = self._alloc(dev, ncell, nf), self._alloc(dev, ncell, nf)
        args = self._cells(dev, temp, ne, chi500) + [self._conv(dev, lam_q, np.float64)]
        check(lib().m3d_optab_sample(self._h, C.c_longlong(ncell), *[ptr(a) for a in args[:3]], C.c_int(nf),
                                     ptr(args[3]), ptr(back), ptr(scat), C.c_uint(DEVICE_PTRS if dev else 0)),
              "m3d_optab_sample")
        return back, scat

    def interpolate_ll(self, temp, ne, chi500, xhat, ehat, lam_q, vproj, chi_scat=None):
        """sample_interpolate_ll: xhat, ehat (and chi_scat when given) (ncell, nf)
        += the table's opacity at the Doppler-shifted wavelength, in place."""
        dev = _is_dev(temp, ne, chi500, lam_q, xhat)
        ncell, nf = int(np.prod(temp.shape)), int(lam_q.shape[0])
        args = self._cells(dev, temp, ne, chi500) + [self._conv(dev, vproj, np.float32),
                                                     self._conv(dev, lam_q, np.float64)]
        check(lib().m3d_optab_sample_ll(self._h, C.c_longlong(ncell), *[ptr(a) for a in args[:4]], C.c_int(nf),
                                        ptr(args[4]), ptr(xhat), ptr(ehat), ptr(chi_scat),
                                        C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_optab_sample_ll")

    def close(self):
        if self._h:
            lib().m3d_optab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _conv(dev, a, dt):
        return a if dev else np.ascontiguousarray(a, dt)

    def _cells(self, dev, temp, ne, chi500):
        return [self._conv(dev, temp, np.float64), self._conv(dev, ne, np.float64), self._conv(dev, chi500, np.float32)]

    @staticmethod
    def _alloc(dev, ncell, nf):
        if dev:
            import torch
            return torch.empty((ncell, nf), dtype=torch.float32, device="cuda")
        return np.empty((ncell, nf), np.float32)

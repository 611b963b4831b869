"""torch.ops.m3d: the library's entry points as PyTorch operators.

load() builds (if needed) and loads libm3d_torch.so (csrc/m3d_torch.cpp), which
registers the operators over the same C ABI as the ctypes front end; they take CUDA
tensors and run on torch's current stream.  The helpers here turn the front end's
atmosphere dicts into the operators' tensor lists.
"""
from __future__ import annotations

import numpy as np

from . import build as _build
from . import lib

_loaded = False

CELL_FIELDS = ("temp", "chi_c", "vx", "vy", "vz", "e_kT", "ne", "tothi", "stark_pe")
SPECIES_FIELDS = ("llam0", "lower_ev", "gpref", "grad", "gw1", "gw2", "gstk", "unsold", "inv_df", "vbar2", "lnbase")
OPS = ("lte_synthesis", "lte_transfer_units", "lte_synthesis_adjoint", "formal_solve", "rotate_array",
       "line_opacity", "integrate_intensity", "qlg_bot_profile", "stateq_update")


def load():
    """Load libm3d_torch.so (building it in-tree when missing or stale); returns torch.ops.m3d."""
    global _loaded
    import torch
    if not _loaded:
        lib()                       # libm3dgpu.so first: the operators call into it
        path = _build.build_torch()
        torch.ops.load_library(path)
        _loaded = True
    return torch.ops.m3d


def atmos_args(atm: dict):
    """(cells, species, shape, slab_nz, geom) of an atmosphere dict whose arrays are
    CUDA tensors (the layout of dispatch_b200.rt.lte_synthesis)."""
    cells = [atm[k].contiguous() for k in CELL_FIELDS]
    species = [sp[k].contiguous() for sp in atm["species"] for k in SPECIES_FIELDS]
    shape = [int(atm["nx"]), int(atm["ny"]), int(atm["nz"])]
    slab_nz = [int(v) for v in atm.get("slab_nz", [atm["nz"]])]
    geom = [float(v) for v in atm.get("ds_cm", (1.0, 1.0, 1.0))] + [float(v) for v in atm.get("ds_code", (1.0, 1.0, 1.0))]
    geom += [float(atm.get("pivot_z", 0.0))] + [float(v) for v in atm.get("ray_offset", (0.0, 0.0))]
    geom += [float(atm.get("tol", 1e-4)), float(atm.get("maser_chi_floor", 1e-4)),
             float(atm.get("maser_dtau_max", 2.0)), float(atm.get("maser_Inu_max", 1e30))]
    return cells, species, shape, slab_nz, geom


def lte_synthesis(atm: dict, nu, llam, vec, wmu, fp64=False, return_itop=False):
    """torch.ops.m3d.lte_synthesis on a device atmosphere: (ie, flux, i_top or None)."""
    ops = load()
    cells, species, shape, slab_nz, geom = atmos_args(atm)
    ie, flux, itop = ops.lte_synthesis(cells, species, shape, slab_nz, geom, nu, llam,
                                       [float(v) for v in np.ravel(vec)], [float(v) for v in np.ravel(wmu)],
                                       bool(fp64), bool(return_itop))
    return ie, flux, (itop if return_itop else None)


def lte_transfer_units(atm: dict, nu, llam, vec, fp64=False):
    ops = load()
    cells, species, shape, _, geom = atmos_args(atm)
    return ops.lte_transfer_units(cells, species, shape, geom, nu, llam, [float(v) for v in np.ravel(vec)],
                                  bool(fp64))


def lte_synthesis_adjoint(atm: dict, nu, llam, vec, wmu, g_flux):
    """The gradient dict of torch.ops.m3d.lte_synthesis_adjoint (the keys of
    dispatch_b200.rt.lte_synthesis_adjoint)."""
    ops = load()
    cells, species, shape, slab_nz, geom = atmos_args(atm)
    g = ops.lte_synthesis_adjoint(cells, species, shape, slab_nz, geom, nu, llam, [float(v) for v in np.ravel(vec)],
                                  [float(v) for v in np.ravel(wmu)], g_flux)
    return dict(zip(("temp", "chi_c", "e_kT", "inv_df", "lnbase", "gpref"), g))

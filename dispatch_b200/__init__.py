"""dispatch_b200 -- B200 (sm_100a) radiative-transfer hot path of OpenMULTI3D.

Python front end of libm3dgpu.so (include/m3dgpu.h), the way tumult and
hopacity reach HOP's libhop.so through cffi (HOP/hopacity/core.py:142-170):
every call returns through a status check that raises M3DError with the
library's message (hop_last_error's role).

Arrays are numpy (host buffers, copied in and out by the library) or torch CUDA
tensors (device pointers, M3D_DEVICE_PTRS, ordered on the library stream).
There is no CPU fallback: without the built library or a GPU the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import build as _build

__all__ = ["M3DError", "lib", "Slab", "LineList", "Species", "Atmos", "init", "LINEAR", "LINEAR2",
           "QUADRATIC", "SHORT_LINEAR", "SHORT_LINEAR2", "BND_MEM", "BND_ZERO", "BND_PCHIP", "BND_LTE",
           "DEVICE_PTRS", "FP64", "GET_PSI", "SPLIT_RATES", "LINE_DIAG", "ROTATE"]

# include/m3dgpu.h
DEVICE_PTRS, FP64, GET_PSI, SPLIT_RATES, LINE_DIAG, ROTATE, AUTOTUNE = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20, 0x40
COL_PERPOINT = 0x80
SE_WARP = 0x100
LINEAR, LINEAR2, QUADRATIC, SHORT_LINEAR, SHORT_LINEAR2 = range(5)
BND_MEM, BND_ZERO, BND_PCHIP, BND_LTE = range(4)

# every symbol include/m3dgpu.h declares
EXPORTS = ("m3d_init", "m3d_free", "m3d_last_error", "m3d_version", "m3d_set_stream", "m3d_synchronize",
           "m3d_launch_count", "m3d_alloc_stats", "m3d_weights", "m3d_qlg_init", "m3d_qlg_tables", "m3d_qlg_bot_profile",
           "m3d_line_opacity", "m3d_lte_background", "m3d_work_to_transfer_units", "m3d_formal_solve",
           "m3d_rotate_array", "m3d_upstream_boundary", "m3d_integrate_intensity", "m3d_lte_synthesis", "m3d_lte_synthesis_windows", "m3d_lte_transfer_units", "m3d_lte_synthesis_adjoint", "m3d_hop_set_state", "m3d_hop_free_state", "m3d_hop_opacity", "m3d_opacity", "m3d_bb_opacity_units", "m3d_h_levels",
           "m3d_profile_enable", "m3d_profile_read", "m3d_rotate_array_noalloc", "m3d_collision_nrows",
           "m3d_collision_rates",
           "m3d_stateq_update", "m3d_ng_accumulate", "m3d_ng_extrapolate", "m3d_bb_damping", "m3d_bf_opacity",
           "m3d_bb_opacity", "m3d_work_to_transfer_units_split", "m3d_bb_rates", "m3d_bf_rates",
           "m3d_integrate_rates", "m3d_normalize_profiles", "m3d_combine_twins", "m3d_update_eta_mask",
           "m3d_lte_populations", "m3d_particle_fields", "m3d_lte_emission", "m3d_col_plan_create",
           "m3d_col_plan_shape", "m3d_stateq_team", "m3d_continuum_opacities",
           "m3d_col_plan_sweep", "m3d_col_plan_fields", "m3d_col_plan_destroy", "m3d_line_opacity_scat", "m3d_chi_scat_units",
           "m3d_long_char_hermite", "m3d_long_char_hermite2", "m3d_short_char_hermite", "m3d_optab_create", "m3d_optab_slopes", "m3d_optab_sample",
           "m3d_optab_sample_ll", "m3d_optab_destroy", "m3d_hydrogen_line", "m3d_h_profile", "m3d_vcs_load", "m3d_vcs_clear",
           "m3d_vcs_supported",
           "m3d_h_opacity", "m3d_save5", "m3d_rcp_check")


class M3DError(RuntimeError):
    pass


class Slab(C.Structure):
    """m3d_slab_t: one depth slab of one ray direction."""

    _fields_ = [("nf", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dir", C.c_int), ("get_psi", C.c_int), ("split_rates", C.c_int), ("pad", C.c_int),
                ("ds", C.c_double * 3), ("vec", C.c_double * 3),
                ("maser_dtau_max", C.c_double), ("maser_Inu_max", C.c_double)]


class LineList(C.Structure):
    """m3d_linelist_t (line_types_mod.f90:22-75)."""

    _fields_ = [("nline", C.c_int), ("llam0", C.c_void_p), ("lower_ev", C.c_void_p),
                ("gpref", C.c_void_p), ("grad", C.c_void_p), ("gw1", C.c_void_p),
                ("gw2", C.c_void_p), ("gstk", C.c_void_p), ("unsold", C.c_void_p),
                ("lev_i", C.c_void_p), ("lev_j", C.c_void_p), ("active", C.c_void_p),
                ("reach_in", C.c_void_p)]


class Species(C.Structure):
    _fields_ = [("ll", LineList), ("inv_df", C.c_void_p), ("vbar2", C.c_void_p), ("lnbase", C.c_void_p)]


class Atmos(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nslab", C.c_int),
                ("slab_nz", C.c_void_p), ("ds_cm", C.c_double * 3), ("ds_code", C.c_double * 3),
                ("pivot_z", C.c_double), ("ray_offset", C.c_double * 2),
                ("temp", C.c_void_p), ("chi_c", C.c_void_p), ("vx", C.c_void_p), ("vy", C.c_void_p),
                ("vz", C.c_void_p), ("e_kT", C.c_void_p), ("ne", C.c_void_p), ("tothi", C.c_void_p),
                ("stark_pe", C.c_void_p), ("nspecies", C.c_int), ("species", C.c_void_p),
                ("tol", C.c_double), ("maser_chi_floor", C.c_double), ("maser_dtau_max", C.c_double),
                ("maser_Inu_max", C.c_double)]


_lib = None


def lib(build: bool = True):
    """Load libm3dgpu.so (building it with nvcc if it is missing or stale)."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if build and (not os.path.exists(path) or _build._stale()):
            _build.build()
        if not os.path.exists(path):
            raise M3DError(f"{path} is not built")
        _lib = C.CDLL(path)
        _lib.m3d_launch_count.restype = C.c_longlong
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib().m3d_last_error(buf, 512)
    return buf.value.decode()


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        raise M3DError(f"{what}: status {rc}: {last_error()}")


# The library keeps one context per host thread (stream, scratch, error string):
# every Python thread that calls it initialises its own.
_tls = threading.local()


def init(device: int = 0) -> None:
    if not getattr(_tls, "initialised", False):
        check(lib().m3d_init(C.c_int(device), C.c_uint(0)), "m3d_init")
        _tls.initialised = True
        _tls.stream = 0


def free() -> None:
    """Release the calling thread's context (m3d_free)."""
    check(lib().m3d_free(), "m3d_free")
    _tls.initialised = False
    _tls.stream = 0


def launch_count() -> int:
    return int(lib().m3d_launch_count())


STAGE_OPACITY, STAGE_SOLVE, STAGE_REDUCE, STAGE_OTHER = range(4)


def profile_enable(on: bool = True) -> None:
    check(lib().m3d_profile_enable(C.c_int(int(on))), "m3d_profile_enable")


def profile_read(stage: int) -> tuple[float, int]:
    ms, n = C.c_double(), C.c_longlong()
    check(lib().m3d_profile_read(C.c_int(stage), C.byref(ms), C.byref(n)), "m3d_profile_read")
    return ms.value, n.value


def synchronize() -> None:
    check(lib().m3d_synchronize(), "m3d_synchronize")


def set_stream(stream_ptr: int | None) -> None:
    """Order the calling thread's library work on this CUDA stream (None: its own stream)."""
    check(lib().m3d_set_stream(C.c_void_p(stream_ptr or 0)), "m3d_set_stream")
    _tls.stream = stream_ptr or 0


def order_after_torch(*arrays) -> None:
    """Device pointers are read and written on the library stream: when torch
    tensors come in, the library moves onto torch's current stream, so that the
    tensors' pending writes come first and torch's later reads see the results."""
    for a in arrays:
        if a is not None and not isinstance(a, np.ndarray) and hasattr(a, "is_cuda") and a.is_cuda:
            import torch
            cur = torch.cuda.current_stream().cuda_stream
            # torch's default stream is the legacy one (handle 0), which the
            # library names by cudaStreamLegacy (0x1); 0 would select its own
            cur = cur if cur != 0 else 1
            if cur != getattr(_tls, "stream", 0):
                set_stream(cur)
            return


def ptr(a) -> C.c_void_p | None:
    """Address of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())


def make_slab(nf, nx, ny, nz, dir, ds, vec, get_psi=False, split_rates=False,
              maser_dtau_max=2.0, maser_Inu_max=1e30) -> Slab:
    s = Slab()
    s.nf, s.nx, s.ny, s.nz, s.dir = nf, nx, ny, nz, dir
    s.get_psi, s.split_rates = int(get_psi), int(split_rates)
    s.ds[:] = [float(v) for v in ds]
    s.vec[:] = [float(v) for v in vec]
    s.maser_dtau_max, s.maser_Inu_max = maser_dtau_max, maser_Inu_max
    return s


from .rt import (formal_solve, rotate_array, upstream_boundary, line_opacity, lte_background,  # noqa: E402
                 work_to_transfer_units, integrate_intensity, qlg_bot_profile, qlg_tables, weights,
                 lte_synthesis, lte_synthesis_windows, lte_transfer_units, lte_synthesis_adjoint, hop_set_state,
                 hop_opacity)
from .stateq import (collision_rates, stateq_update, ng_accumulate, ng_extrapolate, NgState,  # noqa: E402
                     ng_acceleration)

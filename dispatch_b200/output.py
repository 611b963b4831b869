"""The reference's output files written from the library's buffers.

save5 is patch_t%save5 (tasks/patch_mod.f90:4248-4346): one raw float32 array per
patch and window under <run_dir>/save/, named <label>_<key>.bin, with its line in
<label>_meta.txt, which the tumult reader (tumult/io_binary.py) memory-maps.
save_intensity writes the 'ie' and 'flux' arrays of rt_patch_t%save_intensity
(E/SRC/rt_patch_mod.f90:4151-4208) in their shapes: ie (nf, 1, 1, nmu, nset) and
flux (nf, 1, 1, 1, nset).  Arrays are numpy (host) or torch CUDA tensors, given in
numpy order (the reversed Fortran shape).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import DEVICE_PTRS, check, lib, ptr
from .rt import _is_dev


def save5(run_dir: str, label: str, key, mem, add2meta: bool = True) -> None:
    """Write mem (up to 5 axes, numpy order) as the Fortran array of the reversed shape."""
    dev = _is_dev(mem)
    shape = tuple(int(d) for d in mem.shape)[::-1]
    if len(shape) > 5:
        raise ValueError("save5 takes at most 5 axes")
    dims = (C.c_int * 5)(*(list(shape) + [1] * (5 - len(shape))))
    k = [int(v) for v in key]
    arr = mem if dev else np.ascontiguousarray(mem, np.float32)
    check(lib().m3d_save5(str(run_dir).encode(), label.encode(), (C.c_int * len(k))(*k), C.c_int(len(k)), ptr(arr),
                          dims, C.c_int(int(add2meta)), C.c_uint(DEVICE_PTRS if dev else 0)), "m3d_save5")


def save_intensity(run_dir: str, key, ie, flux) -> None:
    """'ie' (nmu, nf) and 'flux' (nf,) of one window and set, as save_intensity lays them out."""
    nmu, nf = ie.shape
    save5(run_dir, "ie", key, ie.reshape(1, nmu, 1, 1, nf))
    save5(run_dir, "flux", key, flux.reshape(1, 1, 1, 1, nf))

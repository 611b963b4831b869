"""m3d_rotate_array_noalloc: rotate_array for callers that cannot let the library
allocate device memory -- a program whose own pool (PyTorch's caching allocator, a
preallocated arena) holds all of it, or whose other streams must not stall on
cudaMalloc/cudaFree.  Its scratch is a fixed 8 MiB array in the library's device
image.  Checked through the C ABI against m3d_rotate_array, bit for bit, on two
calls in a row, with and without a ray offset, and over its size limit; the
library's allocation counter (m3d_alloc_stats) shows that the calls allocate
nothing.  Collected last so that a failure here does not stop a run before the
other tests."""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_noalloc(m, slab, work, ds_code, b2p, off, fp64=False):
    lib = m.lib()
    flags = m.DEVICE_PTRS | (m.FP64 if fp64 else 0)
    offp = None if off is None else (C.c_double * 2)(*off)
    return lib.m3d_rotate_array_noalloc(C.byref(slab), m.ptr(work), (C.c_double * 3)(*ds_code), C.c_double(b2p),
                                        offp, C.c_uint(flags))


def _alloc_stats(m):
    n, sb, tb = C.c_longlong(), C.c_ulonglong(), C.c_ulonglong()
    assert m.lib().m3d_alloc_stats(C.byref(n), C.byref(sb), C.byref(tb)) == 0
    return n.value, sb.value, tb.value


@pytest.mark.parametrize("fp64", [False, True])
def test_noalloc_rotate_matches_rotate_array(m3d, fp64):
    import torch
    cases = [  # (nf, nx, ny, nz, vec, bot2pivot, ray_offset): calls in a row, different shapes
        (8, 24, 20, 5, (0.45, -0.3, math.sqrt(1 - 0.2925)), 2.7, (0.25, -0.5)),
        (32, 120, 120, 3, (-0.61, 0.2, math.sqrt(1 - 0.4121)), 5.1, (0.0, 0.0)),   # 3.7 MB plane in FP64
        (16, 40, 36, 4, (0.2, 0.5, math.sqrt(1 - 0.29)), 1.3, None),               # no ray offset (NULL)
    ]
    rng = np.random.default_rng(12)
    dt = np.float64 if fp64 else np.float32
    for nf, nx, ny, nz, vec, b2p, off in cases:
        work = rng.uniform(0.1, 2.0, (3, nz + 2, ny, nx, nf)).astype(dt)
        a = torch.from_numpy(work).cuda()
        b = a.clone()
        torch.cuda.synchronize()
        slab = m3d.make_slab(nf, nx, ny, nz, 1, [1e7] * 3, vec)
        ds_code = (0.12, 0.1, 0.05)
        # the no-allocation call first, so that no cache grown by m3d_rotate_array
        # could serve it: the library's allocation count stays where it was
        before = _alloc_stats(m3d)
        assert _call_noalloc(m3d, slab, b, ds_code, b2p, off, fp64) == 0, m3d.last_error()
        m3d.synchronize()
        assert _alloc_stats(m3d) == before
        m3d.rotate_array(slab, a, ds_code, b2p, off if off is not None else (0.0, 0.0))
        m3d.synchronize()
        assert torch.equal(a, b)
        assert not torch.equal(b, torch.from_numpy(work).cuda())


def test_noalloc_rejects_planes_over_its_scratch(m3d):
    import torch
    nf, nx, ny, nz = 64, 256, 256, 2          # one plane: 4 Mi floats = 16 MiB > 8 MiB
    work = torch.zeros((3, nz + 2, ny, nx, nf), dtype=torch.float32, device="cuda")
    slab = m3d.make_slab(nf, nx, ny, nz, 1, [1e7] * 3, (0.3, 0.2, math.sqrt(0.87)))
    rc = _call_noalloc(m3d, slab, work, (0.1, 0.1, 0.1), 1.0, (0.0, 0.0))
    assert rc == 1
    assert "exceeds" in m3d.last_error()
    # host buffers would need staging (an allocation): refused before anything runs
    small = m3d.make_slab(4, 6, 5, 2, 1, [1e7] * 3, (0.3, 0.2, math.sqrt(0.87)))
    host = np.zeros((3, 4, 5, 6, 4), np.float32)
    rc = m3d.lib().m3d_rotate_array_noalloc(C.byref(small), m3d.ptr(host), (C.c_double * 3)(0.1, 0.1, 0.1),
                                            C.c_double(1.0), (C.c_double * 2)(0.0, 0.0), C.c_uint(0))
    assert rc == 1
    assert "device pointer" in m3d.last_error()

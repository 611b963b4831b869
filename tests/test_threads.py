"""One library context per host thread.

The reference runs many depth slabs at once on OpenMP threads, each thread owning
one slab (rt_patch_mod.f90:1649-1721 is called per slab task).  The library keeps
its stream, scratch, staging buffers and error string per host thread, so threads
that call it at once do not share host state.  The CPU test checks that errors and
their messages stay in the thread that made them; the GPU test runs four threads
through m3d_formal_solve at the same time, each on its own slab, and checks every
result bit for bit against the oracle."""
import ctypes as C
import math
import threading

import numpy as np
import pytest


def test_errors_stay_in_their_thread(m3d_lib):
    lib = m3d_lib.lib()
    out = {}
    go = threading.Barrier(4)

    def worker(k):
        go.wait()
        # without m3d_init in this thread every call fails with M3D_ENOINIT
        rc = lib.m3d_formal_solve(C.c_int(k % 5), None, None, None, None, None, None, None, None, None, None,
                                  None, C.c_double(0.0), None, C.c_uint(0))
        buf = C.create_string_buffer(256)
        lib.m3d_last_error(buf, 256)
        # a second error, its message naming this thread's own argument
        h = C.create_string_buffer(4096)
        rc2 = lib.m3d_hydrogen_line(C.c_int(k + 1), C.c_int(0), C.c_double(1e15), C.c_uint(0), h)
        buf2 = C.create_string_buffer(256)
        lib.m3d_last_error(buf2, 256)
        n = C.c_longlong(-1)
        lib.m3d_alloc_stats(C.byref(n), None, None)
        out[k] = (rc, buf.value.decode(), rc2, buf2.value.decode(), n.value, lib.m3d_launch_count())

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for k in range(4):
        rc, msg, rc2, msg2, nalloc, launches = out[k]
        assert rc == 3 and "m3d_init" in msg
        assert rc2 == 1 and f"(got {k + 1} -> 0)" in msg2
        assert nalloc == 0 and launches == 0


@pytest.mark.gpu
def test_four_threads_solve_concurrently(m3d, oracle):
    """Four host threads, each with its own context (m3d_init per thread), run the
    quadratic solver with rotate_array and the short-characteristics solver on
    their own slabs at the same time; every result equals the oracle's."""
    import dispatch_b200 as m
    from test_gpu_parity import _slab_case

    nf, nx, ny, nz = 8, 14, 12, 7
    ds = [1.2e7, 1.0e7, 0.8e7]
    cases = []
    for k in range(4):
        vec = np.array([0.3 - 0.1 * k, 0.2 * (k - 1.5) / 1.5, 0.0])
        vec[2] = math.sqrt(1 - (vec[:2] ** 2).sum())
        work, c5, c5u, g5, er, em = _slab_case(100 + k, nf, nx, ny, nz, np.float32, vec)
        solver = ("QUADRATIC", "SHORT_LINEAR")[k % 2]
        cases.append((solver, vec, work))

    def expected(solver, vec, work):
        w = work.copy()
        psi = np.zeros((nz, ny, nx, nf), np.float32)
        slab = oracle.make_slab(nf, nx, ny, nz, 1, ds, vec, get_psi=True)
        oracle.formal_solve(getattr(oracle, solver), slab, w, psi=psi)
        return w, psi

    want = [expected(*c) for c in cases]
    got, errs = {}, {}
    go = threading.Barrier(4)

    def worker(k):
        try:
            m.init(0)                         # this thread's own context
            solver, vec, work = cases[k]
            res = []
            go.wait()
            for _ in range(3):                # several calls, overlapping the other threads'
                w = work.copy()
                psi = np.zeros((nz, ny, nx, nf), np.float32)
                slab = m.make_slab(nf, nx, ny, nz, 1, ds, vec, get_psi=True)
                m.formal_solve(getattr(m, solver), slab, w, psi=psi)
                res.append((w, psi))
            got[k] = res
            m.free()
        except Exception as e:                # noqa: BLE001 -- reported below
            errs[k] = e

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs
    for k in range(4):
        for w, psi in got[k]:
            np.testing.assert_array_equal(w, want[k][0])
            np.testing.assert_array_equal(psi, want[k][1])

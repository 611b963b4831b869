"""The opacity kernels' reciprocal: one Markstein step from the approximate
reciprocal equals the correctly rounded 1/d on every float in [1, 2^126), the range
the kernels' per-line bound keeps 1 + u in; just beyond it (where 1/d is subnormal)
it does not, which is why the kernels bound the argument first."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

ONE, TWO126, TWO127 = 0x3F800000, 0x7E800000, 0x7F000000


def _check(lib, lo, hi):
    n, first = C.c_ulonglong(0), C.c_uint(0)
    rc = lib.m3d_rcp_check(C.c_uint(lo), C.c_uint(hi), C.byref(n), C.byref(first))
    assert rc == 0
    return n.value, first.value


def test_markstein_equals_frcp_rn_on_the_bounded_range(m3d):
    from dispatch_b200 import lib
    n, first = _check(lib(), ONE, TWO126)      # all 2^30 floats in [1, 2^126)
    assert n == 0 and first == 0xFFFFFFFF
    n, first = _check(lib(), TWO126, TWO127)   # reciprocals below 2^-126: flushed
    assert n > 0 and first >= TWO126

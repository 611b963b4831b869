"""The C ABI: libm3dgpu.so builds for sm_100a, loads, and exports exactly what
include/m3dgpu.h declares; no compute call (CPU only)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "m3dgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"^\s*(?:int|long long)\s+(m3d_\w+)\s*\(", src, flags=re.M))


def test_header_matches_python_binding():
    import dispatch_b200 as m
    assert _declared() == set(m.EXPORTS)


def test_library_builds_and_exports_every_symbol():
    from dispatch_b200 import build
    path = build.build()
    lib = C.CDLL(path)
    for name in _declared():
        assert hasattr(lib, name), name


def test_init_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import dispatch_b200 as m
    rc = m.lib().m3d_init(0, 0)
    assert rc != 0
    assert m.last_error()


def test_product_never_reaches_the_oracle():
    """The oracle is test infrastructure: nothing under dispatch_b200/ or include/
    imports, links or names it."""
    for d in ("dispatch_b200", "include"):
        for dirpath, _, files in os.walk(os.path.join(ROOT, d)):
            for f in files:
                if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                    txt = open(os.path.join(dirpath, f)).read()
                    assert "oracle" not in txt, os.path.join(dirpath, f)


def test_oracle_builds(oracle):
    assert os.path.exists(oracle._LIB_PATH)

"""The patch-save files (dispatch_b200.output over m3d_save5): the bytes of the .bin
are the float32 array in Fortran order, the meta lines have patch_t%save_meta's
columns, and the reference's own reader (tumult/io_binary.py, loaded from the
reference tree when it is present) memory-maps them back to the same arrays."""
import os
import sys
import types

import numpy as np
import pytest

# the reference's OpenMULTI3D tree (experiments/OpenMULTI3D), where a machine has it;
# the reader test skips without it
REF = os.environ.get("M3D_REFERENCE_ROOT", "")


def _read_meta(folder, label):
    lines = open(os.path.join(folder, f"{label}_meta.txt")).read().splitlines()
    return lines[0], [ln for ln in lines[1:]]


def test_save5_layout(m3d_lib, tmp_path):
    from dispatch_b200 import output
    rng = np.random.default_rng(0)
    ie = rng.random((3, 1, 1, 1, 17)).astype(np.float32)          # numpy order of (17, 1, 1, 1, 3)
    output.save5(str(tmp_path), "ie", (1, 2, 3), ie)
    output.save5(str(tmp_path), "ie", (1, 2, 4), 2 * ie)
    output.save5(str(tmp_path), "flux", (5, 12), ie[:1])
    folder = os.path.join(str(tmp_path), "save")
    head, rows = _read_meta(folder, "ie")
    assert head == "* filename" + " " * 21 + "bytes"
    assert rows[0] == f"{'ie_001002003.bin':<32}{32:4d}" + "".join(f"{d:10d}" for d in (17, 1, 1, 1, 3))
    assert rows[1].startswith("ie_001002004.bin ")
    raw = np.fromfile(os.path.join(folder, "ie_001002003.bin"), np.float32)
    np.testing.assert_array_equal(raw, ie.ravel())        # numpy C order == Fortran order of the reversed shape
    assert os.path.exists(os.path.join(folder, "flux_005012.bin"))
    with pytest.raises(m3d_lib.M3DError, match="not associated"):
        output.save5(str(tmp_path), "empty", (1, 1), np.zeros((0, 4), np.float32))


def test_reference_reader_reads_them(m3d_lib, tmp_path):
    if not REF or not os.path.isdir(os.path.join(REF, "tumult")):
        pytest.skip("the reference's tumult package is not present")
    pkg = types.ModuleType("tumult")
    pkg.__path__ = [os.path.join(REF, "tumult")]
    saved = sys.modules.get("tumult")
    sys.modules["tumult"] = pkg
    try:
        import importlib
        io_binary = importlib.import_module("tumult.io_binary")
        from dispatch_b200 import output
        rng = np.random.default_rng(1)
        nmu, nf = 5, 24
        parts = {}
        for inu in (1, 2, 3):
            ie = rng.random((nmu, nf)).astype(np.float32)
            flux = rng.random(nf).astype(np.float32)
            output.save_intensity(str(tmp_path), (1, inu), ie, flux)
            parts[inu] = (ie, flux)
        dct, dims = io_binary.load_patch_files(os.path.join(str(tmp_path), "save"), "ie")
        assert dims == (nf, 1, 1, nmu, 1)
        for inu, (ie, flux) in parts.items():
            np.testing.assert_array_equal(np.asarray(dct[(1, inu)])[:, 0, 0, :, 0], ie.T)
        full = io_binary.read_patch_save(os.path.join(str(tmp_path), "save"), "flux", n_windows=3, lazy=False,
                                         fdim=0)
        np.testing.assert_array_equal(np.asarray(full[0])[:, 0, 0, 0, 0],
                                      np.concatenate([parts[i][1] for i in (1, 2, 3)]))
    finally:
        if saved is None:
            sys.modules.pop("tumult", None)
        else:
            sys.modules["tumult"] = saved
        for k in [k for k in sys.modules if k.startswith("tumult.")]:
            sys.modules.pop(k)

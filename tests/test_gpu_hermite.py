"""long_char_hermite on the device against the oracle (bit for bit, FP32): both
directions, the ghost's state given or the zeroed ghost's secant step, with and
without the Lambda diagonal."""
import numpy as np
import pytest

from hermite_cases import slab_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dir", [1, -1])
@pytest.mark.parametrize("ghost", [True, False])
@pytest.mark.parametrize("psi_on", [True, False])
def test_long_char_hermite_bit_exact(m3d, oracle, dir, ghost, psi_on):
    work, fld, ghosts, ds = slab_case(seed=5 + dir)
    nz, ny, nx, nf = work.shape[1] - 2, work.shape[2], work.shape[3], work.shape[4]
    vec = np.array([0.3, -0.2, 0.0])
    vec[2] = dir * np.sqrt(1 - 0.13)
    g = ghosts["bottom" if dir > 0 else "top"] if ghost else None
    out = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        w = work.copy()
        zg = 0 if dir > 0 else nz + 1
        if not ghost:
            w[:, zg] = 0.0                    # the zeroed ghost of set_upstream_boundary's top branch
        else:
            w[2, zg] = w[1, zg]               # the LTE ghost: Inu = Snu
        psi = np.zeros((nz, ny, nx, nf), np.float32)
        slab = mod.make_slab(nf, nx, ny, nz, dir, [ds * 1.5, ds * 1.5, ds], vec, get_psi=psi_on)
        args = [fld[k] for k in ("beta", "pe", "dpe_dz", "dlnt_dz", "temp", "hknu")]
        if name == "o":
            oracle.long_char_hermite(slab, w, psi, *args, ghost=g)
        else:
            m3d.rt.long_char_hermite(slab, w, psi, *args, ghost=g)
        out[name] = (w, psi)
    np.testing.assert_array_equal(out["g"][0], out["o"][0])
    np.testing.assert_array_equal(out["g"][1], out["o"][1])
    assert np.isfinite(out["o"][0]).all()
    if psi_on:
        assert out["o"][1].max() > 0


def test_long_char_hermite_rejects_thin_slab(m3d):
    work, fld, ghosts, ds = slab_case(nz=2)
    slab = m3d.make_slab(work.shape[4], work.shape[3], work.shape[2], 2, 1, [ds] * 3, [0, 0, 1.0])
    with pytest.raises(m3d.M3DError, match="nz >= 3"):
        m3d.rt.long_char_hermite(slab, work, None, *[fld[k] for k in ("beta", "pe", "dpe_dz", "dlnt_dz", "temp",
                                                                       "hknu")])

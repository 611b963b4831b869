"""m3d_h_levels (init_H_levels with compute_shield) on the B200 against the oracle:
shield, the level populations and the occupation probabilities, with and without
occupation probabilities (the dissolved levels too).  The device's double exp and pow
may differ from glibc's in the last place: 1e-12 relative."""
import numpy as np
import pytest

from dispatch_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("occupation", [True, False])
def test_h_levels_match_oracle(m3d, oracle, occupation):
    import torch
    from oracle import continuum as oc
    from dispatch_b200.continuum import h_levels
    _, _, _, cells = synth.continuum_case(ncell=5000, nlam=8)
    cells = dict(cells)
    cells["dxi"] = cells["dxi"].copy()
    cells["dxi"][::7] = 0.0
    cells["dxi"][0] = 0.03
    so, lo, wo = oc.h_levels(cells, 16, occupation)
    sg, lg, wg = h_levels(cells, 16, occupation)
    np.testing.assert_allclose(sg, so, rtol=1e-12)
    np.testing.assert_allclose(lg, lo, rtol=1e-12, atol=0)
    assert np.array_equal(lg == 0, lo == 0)
    if occupation:
        np.testing.assert_allclose(wg, wo, rtol=1e-12)
    else:
        assert wg is None and np.any(lo == 0)
    # device pointers give the same
    dev = {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
           for k, v in cells.items()}
    sd, ld, wd = h_levels(dev, 16, occupation)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sd.cpu().numpy(), sg)
    np.testing.assert_array_equal(ld.cpu().numpy(), lg)


def test_h_levels_feed_the_occupation_continuum(m3d, oracle):
    """The levels from m3d_h_levels as the 'H BF' components' populations and
    occupation probabilities: the continuum from them equals the oracle's on the same
    inputs bit for bit."""
    from oracle import continuum as oc
    from dispatch_b200.continuum import continuum_opacities, h_levels
    comps, lam, nu, cells = synth.continuum_case(ncell=2000, nlam=128)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")} | {"nHI": cells["nHI"]}
    sh, ln, lw = h_levels(cells, 8, True)
    cells["shield"] = sh
    occ = []
    for c in comps[12:]:
        c = dict(c)
        i = c["level_i"]
        c["level_n"], c["level_w"] = ln[i - 1], lw[i - 1]
        occ.append(c)
    cells_nohrest = {k: v for k, v in cells.items() if k != "nHI"}
    xo, _ = oc.continuum_opacities(occ, lam, nu, cells_nohrest, sigma=False)
    xg, _ = continuum_opacities(occ, lam, nu, cells_nohrest, sigma=False)
    assert xo.max() > 0
    np.testing.assert_array_equal(xg, xo)

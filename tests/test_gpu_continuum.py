"""The continuum opacity on the B200 (m3d_continuum_opacities) against the oracle
(oracle/or_continuum.c) on the seeded case of synth.continuum_case: fourteen
components of every absorption-factor kind and interpolation form, two 'H BF'
levels under occupation probabilities (wcalc2) among them, a visible and an
ultraviolet window (the Rayleigh cut at 1400 A, tables covering the window in part).

Bit-exact wherever both sides do the same IEEE operations: the interpolations, the
absorption factors without exponentials, the reference's own exp4, electron and
Rayleigh scattering.  Where the reference calls the platform's exp or log (the
H-rest and H FF factors and a level's Boltzmann factor in double, the Boltzmann
factor beta, a table logarithmic in wavelength only, the exp of a temperature-free
logarithmic table), the device's functions may differ from glibc's in the last place:
there the results agree to 1e-6 relative (3e-6 where a row's logarithm is
exponentiated again) and nearly all of them bit for bit.
"""
import numpy as np
import pytest

from dispatch_b200 import synth

pytestmark = pytest.mark.gpu

WINDOWS = ((3500.0, 12000.0), (1000.0, 3000.0))


@pytest.fixture(scope="module")
def oc(oracle):
    from oracle import continuum
    return continuum


def _exact(comps, cells):
    """The components and cells whose arithmetic calls no platform exp or log."""
    from dispatch_b200 import continuum as cn
    keep = []
    for c in comps:
        if c["kind"] in (cn.H_FF, cn.REGULAR):
            continue
        if c["ilogl"] and not c["log_table"]:
            continue                                        # log of the interpolated row
        if c["tt"].size == 1 and c["ilogl"]:
            continue                                        # exp of the wavelength interpolation
        keep.append(c)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}   # the H rest's exps
    return keep, cells


@pytest.mark.parametrize("window", WINDOWS)
def test_continuum_matches_oracle(m3d, oc, window):
    from dispatch_b200.continuum import continuum_opacities
    comps, lam, nu, cells = synth.continuum_case(ncell=3000, nlam=256, lam_range=window)
    xo, so = oc.continuum_opacities(comps, lam, nu, cells)
    xg, sg = continuum_opacities(comps, lam, nu, cells)
    assert np.all(np.isfinite(xg)) and xg.max() > 0
    np.testing.assert_allclose(xg, xo, rtol=1e-6, atol=0)
    np.testing.assert_array_equal(sg, so)
    assert np.mean(xg == xo) > 0.95
    # the same without any platform exp or log: bit for bit
    ce, celle = _exact(comps, cells)
    assert len(ce) >= 6
    beta = np.random.default_rng(9).uniform(1e-6, 0.8, (3000, 256)).astype(np.float32)
    xo, so = oc.continuum_opacities(ce, lam, nu, celle, beta=beta)
    xg, sg = continuum_opacities(ce, lam, nu, celle, beta=beta)
    np.testing.assert_array_equal(xg, xo)
    np.testing.assert_array_equal(sg, so)


def test_continuum_each_component_bit_exact_or_to_the_ulp(m3d, oc):
    """Component by component (the order of the sum is the reference's), with the
    beta the oracle forms from nu."""
    from dispatch_b200.continuum import continuum_opacities
    comps, lam, nu, cells = synth.continuum_case(ncell=500, nlam=128)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}
    exact_kinds = {1, 2, 5, 6, 7, 8, 9}
    for j, c in enumerate(comps):
        xo, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
        xg, _ = continuum_opacities([c], lam, nu, cells, sigma=False)
        assert xo.max() > 0, j
        plain = (c["kind"] in exact_kinds or c.get("occupation")) and not c.get("istim") \
            and not (c["ilogl"] and not c["log_table"]) and not (c["tt"].size == 1 and c["ilogl"])
        if plain:
            np.testing.assert_array_equal(xg, xo, err_msg=f"component {j}")
        else:
            # a table logarithmic in wavelength only takes the log of each interpolated
            # row: one last-place difference of the log (|ln y| up to ~14 here) moves the
            # exponentiated result by up to ~1.5e-6 relative
            np.testing.assert_allclose(xg, xo, rtol=3e-6, atol=0, err_msg=f"component {j}")


def test_continuum_device_pointers(m3d, oc):
    import torch
    from dispatch_b200.continuum import continuum_opacities
    comps, lam, nu, cells = synth.continuum_case(ncell=1000, nlam=64)
    xh, sh = continuum_opacities(comps, lam, nu, cells)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dc = {k: (dev(v) if isinstance(v, np.ndarray) else v) for k, v in cells.items()}
    dcomps = [{k: (dev(v) if k in ("n", "n2", "part", "level_n", "level_w") else v) for k, v in c.items()}
              for c in comps]
    xd, sd = continuum_opacities(dcomps, lam, nu, dc)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(xd.cpu().numpy(), xh)
    np.testing.assert_array_equal(sd.cpu().numpy(), sh)


def test_continuum_rejects(m3d):
    from dispatch_b200.continuum import continuum_opacities
    comps, lam, nu, cells = synth.continuum_case(ncell=10, nlam=16)
    bad = dict(comps[0])
    bad["kind"] = 0
    with pytest.raises(m3d.M3DError, match="unknown kind"):
        continuum_opacities([bad], lam, nu, cells)
    bad = dict(comps[3])
    bad.pop("part")
    with pytest.raises(m3d.M3DError, match="NULL density"):
        continuum_opacities([bad], lam, nu, cells)
    with pytest.raises(m3d.M3DError, match="beta or nu"):
        continuum_opacities([comps[10]], lam, None, cells)
    nosh = {k: v for k, v in cells.items() if k != "shield"}
    with pytest.raises(m3d.M3DError, match="occupation"):
        continuum_opacities([comps[12]], lam, nu, nosh)
    bad = dict(comps[12])
    bad.pop("level_w")
    with pytest.raises(m3d.M3DError, match="NULL density"):
        continuum_opacities([bad], lam, nu, cells)


def test_continuum_h_occupation_levels(m3d, oc):
    """The 'H BF' levels under occupation probabilities alone (no H rest), both
    wavelength classes of wcalc2 and dissolved_only, bit for bit; and the same level
    with its table given temperature nodes keeps absorption_factor's huge(1d0)."""
    from dispatch_b200.continuum import continuum_opacities
    comps, lam, nu, cells = synth.continuum_case(ncell=2000, nlam=256)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}
    for c in comps[12:]:
        xo, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
        xg, _ = continuum_opacities([c], lam, nu, cells, sigma=False)
        assert (xo > 0).mean() > 0.2
        np.testing.assert_array_equal(xg, xo)
    c = dict(comps[12])
    c["tt"] = np.array([5000.0, 8000.0])
    c["xkap"] = np.vstack([c["xkap"], c["xkap"]])
    xo, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
    xg, _ = continuum_opacities([c], lam, nu, cells, sigma=False)
    np.testing.assert_array_equal(xg, xo)

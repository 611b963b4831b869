"""The continuum-opacity oracle (oracle/or_continuum.c) against what the reference
states and against independent restatements:

* load_lam_interp_weights' stencils bracket each wavelength, the weights sum to one,
  and wavelengths outside a table that may not be extrapolated get none;
* a table constant in wavelength and temperature is reproduced, one linear in
  wavelength too, to the rounding of the real(4) weights, in every interpolation form;
* set_table's stored form (dispatch_b200.continuum.set_table) against its formula;
* the Thomson constant against const_mod's sigma_th, electron and Rayleigh
  scattering and the H rest against direct numpy forms;
* components tabulated with stimulated emission end up divided by 1 - beta;
* an 'H BF' level under occupation probabilities (wcalc2, level_mod.f90:149-279)
  against an independent float32 restatement, and in the limit without perturbers
  (w = wstar = 1) against the same level without occupation probabilities.
"""
import numpy as np
import pytest

from dispatch_b200 import synth
from dispatch_b200.continuum import HMINUS, set_table


@pytest.fixture(scope="module")
def oc(oracle):
    from oracle import continuum
    return continuum


def _flat(value, lam_lo, lam_hi, nnu=12, tnodes=(4000.0, 7000.0, 10000.0), **kw):
    tl = np.geomspace(lam_lo, lam_hi, nnu)
    raw = np.full((len(tnodes), nnu), value)
    xk, scale, logt = set_table(raw, kw.pop("ilogt", False), kw.get("ilogl", False))
    c = {"kind": HMINUS, "lam": tl, "tt": np.asarray(tnodes), "xkap": xk, "xkap_scale": scale, "log_table": logt,
         "minl": tl[0], "maxl": tl[-1], "mint": 0.0, "maxt": 1e9}
    c.update(kw)
    return c


def _cells(ncell=40, seed=1):
    rng = np.random.default_rng(seed)
    t = rng.uniform(3000.0, 11000.0, ncell)
    ne = 10.0 ** rng.uniform(10, 14, ncell)
    return {"temp": t, "teta": 5040.0 / t, "e_kT": synth.EE / (synth.BK * t), "pe": ne * synth.BK * t,
            "dxi": np.zeros(ncell), "ne": ne, "helium_scattering": True}


def test_weights_bracket_and_sum(oc):
    comps, lam, nu, cells = synth.continuum_case(ncell=8, nlam=300, lam_range=(2000.0, 20000.0))
    for c in comps:
        act, iw, quad, lag, fs, fe = oc.bf_weights(c, lam)
        tl = c["lam"]
        inside = (lam >= tl[0]) & (lam <= tl[-1])
        allowed = inside | ((lam > tl[-1]) & bool(c.get("maxex"))) | ((lam < tl[0]) & bool(c.get("minex")))
        assert act == bool(allowed.any())
        assert np.array_equal(iw >= 0, allowed)
        if not act:
            continue
        idx = np.flatnonzero(allowed)
        assert fs == idx[0] and fe == idx[-1]
        for f in idx:
            w = lag[f, :3 if quad[f] else 2].astype(np.float64)
            assert w.sum() == pytest.approx(1.0, abs=2e-7 * np.abs(w).sum())   # real(4) weights
            if inside[f] and not quad[f]:
                j = iw[f]
                assert tl[j] <= lam[f] <= tl[j + 1]
            if quad[f]:
                assert not c["ldisk"][iw[f]]


def test_constant_table_reproduced(oc):
    cells = _cells()
    lam = np.geomspace(4000.0, 9000.0, 50)
    n = 10.0 ** np.random.default_rng(2).uniform(8, 11, 40)
    forms = ({}, {"kvadt": True}, {"kvadl": True}, {"ilogt": True}, {"ilogl": True}, {"ilogl": True, "ilogt": True})
    for kw in forms:
        c = _flat(3e-17, 3000.0, 10000.0, n=n, **kw)
        xhat, _ = oc.continuum_opacities([c], lam, None, cells, sigma=False)
        want = (n * c["xkap_scale"]).astype(np.float32)
        # the stored table is 1 (or ln 1 = 0) everywhere: the interpolation returns it,
        # to the rounding of its real(4) weights, whose sum is 1 only to an ulp or two
        np.testing.assert_allclose(xhat, np.repeat(want[:, None], lam.size, axis=1), rtol=4e-7, err_msg=str(kw))


def test_linear_table_to_rounding(oc):
    cells = _cells()
    lam = np.geomspace(4100.0, 8900.0, 77)
    tl = np.linspace(4000.0, 9000.0, 21)
    raw = np.tile(1.0 + (tl - 4000.0) / 5000.0, (3, 1))
    xk, scale, logt = set_table(raw, False, False)
    c = {"kind": HMINUS, "lam": tl, "tt": np.array([4000.0, 7000.0, 10000.0]), "xkap": xk, "xkap_scale": scale,
         "log_table": logt, "minl": tl[0], "maxl": tl[-1], "mint": 0.0, "maxt": 1e9, "kvadl": True,
         "n": np.ones(40)}
    xhat, _ = oc.continuum_opacities([c], lam, None, cells, sigma=False)
    np.testing.assert_allclose(xhat, np.tile(1.0 + (lam - 4000.0) / 5000.0, (40, 1)), rtol=2e-6)


def test_set_table_form():
    raw = np.array([[1e-30, 2e-30, 0.0], [4e-30, 8e-30, 1e-30]])
    xk, scale, logt = set_table(raw, True, False)
    assert logt and scale == 8e-30
    np.testing.assert_array_equal(xk, (np.log(np.where(raw > 0, raw, 1e-37)) - np.log(8e-30)).astype(np.float32))
    xk, scale, logt = set_table(raw[:1], True, False)   # no temperature dependence: ilogl decides
    assert not logt and scale == 2e-30
    np.testing.assert_array_equal(xk, (raw[:1] / 2e-30).astype(np.float32))


def test_scattering_and_hrest(oc):
    cells = _cells()
    cells.update(nHI=10.0 ** np.linspace(14, 17, 40), partHI=np.full(40, np.log(2.0)), nHeI=np.full(40, 1e15),
                 nH2=np.full(40, 1e10), HI_xion=13.598434, dxi=np.linspace(0, 0.05, 40))
    lam = np.concatenate([np.geomspace(1000.0, 1399.0, 20), np.geomspace(1401.0, 12000.0, 60)])
    xhat, sg = oc.continuum_opacities([], lam, None, cells)
    # Thomson: const_mod's sigma_th = 8/3 pi e^4/(m^2 c^4) = 6.6524e-25 cm^2
    thomson = float(8.0 / 3.0 * 3.14159265359) * (4.80325e-10**2 / (9.109534e-28 * 2.99792458e10**2))**2
    assert thomson == pytest.approx(6.6524e-25, rel=1e-4)
    xr = np.where(lam > 1400.0, 1.0 / np.maximum(1026.0, lam) ** 2, 0.0)
    rayh = (5.799e-13 + xr * (1.422e-6 + xr * 2.784))[None, :] * cells["nHI"][:, None]
    rayh2 = (8.14e-13 + xr * (1.28e-6 + xr * 1.61))[None, :] * 1e10
    he = 0.66520e-24 * 4.0 * (500.0 / lam) ** 4
    want = thomson * cells["ne"][:, None] + (rayh + rayh2) * xr**2 + he[None, :] * 1e15
    np.testing.assert_allclose(sg, want, rtol=3e-7)
    # the H rest: the hydrogenic levels above n = 15 up to the lowered limit
    ekt, dxi = cells["e_kT"], cells["dxi"]
    fakt = np.exp(-ekt * (13.598434 - dxi) - np.log(2.0)) * 2.0898e-26 / (2 * 13.598434 * ekt) * cells["nHI"]
    hr = fakt * (np.exp(ekt * (13.598434 / 240.25 - dxi)) - 1)
    hr = np.where(13.598434 >= 240.25 * dxi, hr, 0.0)
    np.testing.assert_allclose(xhat, hr[:, None] * lam[None, :] ** 3, rtol=3e-7)


def test_stimulated_components_over_one_minus_beta(oc):
    comps, lam, nu, cells = synth.continuum_case(ncell=30, nlam=40)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}   # no H rest: the component alone
    c = dict(comps[0])
    beta = np.random.default_rng(4).uniform(1e-6, 0.7, (30, 40)).astype(np.float32)
    plain, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
    c["istim"] = True
    stim, _ = oc.continuum_opacities([c], lam, nu, cells, beta=beta, sigma=False)
    np.testing.assert_array_equal(stim, plain / (np.float32(1.0) - beta))


def test_full_case_finite(oc):
    comps, lam, nu, cells = synth.continuum_case(ncell=200, nlam=128)
    xhat, sg = oc.continuum_opacities(comps, lam, nu, cells)
    assert np.all(np.isfinite(xhat)) and np.all(xhat > 0) and np.all(sg > 0)
    # each kind contributes somewhere
    for k, c in enumerate(comps):
        x1, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
        assert x1.max() > 0, k


def _wcalc2_numpy(c, lam, cells, fs, fe, ab):
    """wcalc2 restated with numpy scalars in the kinds of level_mod.f90:149-279:
    real(8) set-up per wavelength, real(4) arithmetic per cell; exp_neg0 is the
    oracle's K0 function (pinned by tests/test_oracle_contracts.py)."""
    from oracle.oracle import exp_neg0
    f32 = np.float32
    hh, ee, cc, ryd = 6.626176e-27, 1.602189e-12, 2.99792458e10, 13.598434
    li = int(c["level_i"])
    redcut = (hh * cc / ee) / ((float(li) ** -2.0 - float(li + 1) ** -2.0) * ryd) * 1e8
    q = f32(2.0898e-26) / f32(2 * li ** 5)
    ncell = cells["ne"].size
    out = np.zeros((ncell, lam.size), np.float32)
    for f in range(fs, fe + 1):
        cutfac = np.exp((redcut - lam[f]) * 1e-2) if lam[f] > redcut else 1.0
        if not cutfac > 0.1:
            continue
        g = f32(float(q) * cutfac * float(ab[f]))
        nu = cc / lam[f] * float(f32(1e8))
        ns = 1.0 - (c["level_xion"] + (hh / ee) * nu) / ryd
        w = c["level_w"].astype(np.float32)
        n = c["level_n"].astype(np.float32)
        if ns > 0:
            ns = 1.0 / np.sqrt(ns)
            ns2 = ns * ns
            rih = ns * np.sqrt(2.5 * ns2 + 0.5)
            t1 = 5.29177349e-9 * (rih + float(f32(1.73)))
            t2 = 5.29177349e-9 * (rih + float(f32(1.02)))
            k = float(f32(8.3e14)) / (ns2 * ns2)
            if ns > 3.0:
                k = k * float(f32(5.33333333)) * ns / ((ns + 1.0) * (ns + 1.0))
            kd = k * np.sqrt(k)
            x1, x2, kk = f32(t1 * t1 * t1), f32(t2 * t2 * t2), f32(kd)
            nh43 = (4.18879 * c["n"]).astype(np.float32)
            nhe43 = (4.18879 * cells["nHeI"]).astype(np.float32)
            a = nh43 * x1 + nhe43 * x2
            E, omE = exp_neg0(a)
            xs = cells["shield"].astype(np.float32)
            xk = xs * kk
            ne1 = cells["ne"].astype(np.float32)
            frac = f32(0.1402) * xk * kk / (ne1 * (f32(1.0) + f32(0.1285) * xk))
            charged = cells["shield"] * kd < 1e4
            C = np.where(charged, frac / (f32(1.0) + frac), f32(1.0)).astype(np.float32)
            omC = np.where(charged, f32(1.0) / (f32(1.0) + frac), f32(0.0)).astype(np.float32)
            omw = (1.0 - c["level_w"]).astype(np.float32)
            d = np.where(w > f32(0.5), (omE + E * omC) - omw, w - E * C).astype(np.float32)
            out[:, f] = d * n * g
        elif not c.get("dissolved_only"):
            out[:, f] = w * n * g
    return out


def test_h_occupation_level_against_numpy(oc):
    comps, lam, nu, cells = synth.continuum_case(ncell=60, nlam=120)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}
    for c in comps[12:]:
        assert c["occupation"] and c["tt"].size == 1
        act, iw, quad, lag, fs, fe = oc.bf_weights(c, lam)
        assert act
        # interp_xkap_2's table at the window, lam^3, times real(xkap_scale, 4)
        ab = np.zeros(lam.size, np.float32)
        xk = c["xkap"][0]
        for f in range(fs, fe + 1):
            if iw[f] < 0:
                continue
            v = np.float32(0.0) + xk[iw[f]] * lag[f, 0]
            v = v + xk[iw[f] + 1] * lag[f, 1]
            if quad[f]:
                v = v + xk[iw[f] + 2] * lag[f, 2]
            ab[f] = v * np.float32(lam[f] ** 3) * np.float32(c["xkap_scale"])
        want = _wcalc2_numpy(c, lam, cells, fs, fe, ab)
        got, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
        assert (want > 0).mean() > 0.2
        np.testing.assert_array_equal(got, want)


def test_h_occupation_without_perturbers(oc):
    """No neutral perturbers and the charged term out of reach: wstar = 1 and w = 1,
    so the dissolved states add nothing and beyond the limit the level adds its plain
    bound-free opacity (to the rounding of the two products' orders)."""
    comps, lam, nu, cells = synth.continuum_case(ncell=40, nlam=200)
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}
    cells["nHeI"] = np.zeros(40)
    cells["shield"] = np.full(40, 1e10)
    c = dict(comps[12])
    c["n"] = np.zeros(40)
    c["level_w"] = np.ones(40)
    occ, _ = oc.continuum_opacities([c], lam, nu, cells, sigma=False)
    plain = dict(c)
    plain["occupation"] = False
    ref, _ = oc.continuum_opacities([plain], lam, nu, cells, sigma=False)
    edge = 911.267 * 4
    below, beyond = lam > edge * 1.001, lam < edge * 0.999
    assert np.all(occ[:, below] == 0)
    np.testing.assert_allclose(occ[:, beyond], ref[:, beyond], rtol=1e-6)


def test_h_levels(oc):
    """init_H_levels: with occupation probabilities the populations are nHI g exp(..)/Z
    with Z = sum w g exp(..), so sum_i w_i n_i = nHI; without, nHI g exp(..) exp(-ln U)
    and the levels above n = sqrt(RYD/dxi) dissolved; the shielding as stated."""
    _, _, _, cells = synth.continuum_case(ncell=200, nlam=8)
    sh, ln, lw = oc.h_levels(cells, 12, occupation=True)
    want = (np.float64(np.float32(0.08989)) * cells["ne"] ** 0.16667 / np.sqrt(cells["temp"]))
    np.testing.assert_allclose(sh, (1.0 + want) ** 3.15 / cells["ne"], rtol=1e-14)
    np.testing.assert_allclose((lw * ln).sum(axis=0), cells["nHI"], rtol=1e-13)
    assert np.all((lw > 0) & (lw <= 1)) and np.all(np.diff(lw, axis=0) <= 0)   # higher levels dissolve more
    cells2 = dict(cells)
    cells2["dxi"] = np.where(np.arange(200) % 5 == 0, 0.0, 0.02 + 0.1 * np.random.default_rng(1).random(200))
    cells2["dxi"][0] = 0.05
    sh2, ln2, lw2 = oc.h_levels(cells2, 12, occupation=False)
    assert lw2 is None
    i = np.arange(1, 13)[:, None]
    xion = 13.598434 * (np.float32(1) - np.float32(1) / (i * i).astype(np.float32)).astype(np.float64)
    full = cells["nHI"] * (2.0 * i * i * np.exp(-cells["e_kT"] * xion)) * np.exp(-cells["partHI"])
    nniv = np.where(cells2["dxi"] > 0, np.floor(np.sqrt(13.598434 / np.where(cells2["dxi"] > 0, cells2["dxi"], 1))), 99)
    assert np.all(ln2[i[:, 0][:, None] > nniv[None, :]] == 0)
    keep = i <= nniv[None, :] - 1
    np.testing.assert_allclose(ln2[keep], full[keep], rtol=1e-13)
    np.testing.assert_allclose(ln2[:, cells2["dxi"] == 0], full[:, cells2["dxi"] == 0], rtol=1e-13)

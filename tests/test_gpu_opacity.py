"""m3d_opacity: composition_type%opacity's pipeline (composition_mod.f90:3122-3260) --
the continuum in the working form, the line list of the loaded state against it as
the tolerance reference, chi = xhat - ehat beta (+ scat) -- against the same
composition of the oracle's continuum_opacities and add_opacity_equi.  Bit for bit
where the continuum calls no platform exp or log and beta is given; with beta from
nu and every component, to the device's exp/log (1e-5 relative)."""
import numpy as np
import pytest

from dispatch_b200 import synth

pytestmark = pytest.mark.gpu


def _case():
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=48, window=3)
    ncell = atm["temp"].size
    lam = np.exp(llam)
    comps, _, _, cells = synth.continuum_case(ncell=ncell, nlam=8)
    nu = synth.HZ_TO_AA / lam
    return atm, lam, nu, llam, comps, cells


def _oracle(oracle, oc, atm, lam, nu, llam, comps, cells, beta, margin, llist=True, disjoint=False):
    xo, so = oc.continuum_opacities(comps, lam, nu, cells, beta=beta)
    ncell = xo.shape[0]
    chil = np.zeros_like(xo)
    etal = np.zeros_like(xo)
    if llist:
        lo, hi = llam[0] - margin / lam[0], llam[-1] + margin / lam[0]
        for sp0 in atm["species"]:
            sp = dict(sp0)
            sp["active"] = ((sp["llam0"] >= lo) & (sp["llam0"] <= hi)).astype(np.uint8)
            cl = {"vproj": np.zeros(ncell, np.float32), "inv_df": sp["inv_df"], "vbar2": sp["vbar2"],
                  "lnbase": sp["lnbase"], "e_kT": atm["e_kT"], "ne": atm["ne"], "tothi": atm["tothi"],
                  "stark_pe": atm["stark_pe"]}
            oracle.add_opacity_equi(sp, llam, chil, etal, xo, oracle.logref(xo), cl)
        chi = (xo + chil) - (xo + etal) * beta
    else:
        chi = xo * (np.float32(1.0) - beta)
    if not disjoint:
        chi = chi + so
    return chi.astype(np.float32), so


def test_opacity_matches_oracle_bit_exact(m3d, oracle):
    from oracle import continuum as oc
    from dispatch_b200.continuum import opacity
    atm, lam, nu, llam, comps, cells = _case()
    # the components and cells that call no platform exp or log, beta given
    comps = [c for c in comps if c["kind"] not in (4, 10) and not (c["ilogl"] and not c["log_table"])
             and not (c["tt"].size == 1 and c["ilogl"])]
    cells = {k: v for k, v in cells.items() if k not in ("nHI", "partHI")}
    ncell = atm["temp"].size
    beta = np.random.default_rng(3).uniform(1e-6, 0.6, (ncell, lam.size)).astype(np.float32)
    m3d.hop_set_state(atm)
    for llist, disjoint in ((True, False), (True, True), (False, False)):
        chi, scat = opacity(comps, lam, nu, cells, beta=beta, include_llist=llist, line_margin=0.3,
                            disjoint=disjoint)
        want, so = _oracle(oracle, oc, atm, lam, nu, llam, comps, cells, beta, 0.3, llist, disjoint)
        np.testing.assert_array_equal(scat, so)
        np.testing.assert_array_equal(chi, want, err_msg=f"llist={llist} disjoint={disjoint}")
    # the lines add to the continuum (where a point has none, xhat - xhat beta and
    # xhat (1 - beta) may round an ulp apart)
    c0, _ = opacity(comps, lam, nu, cells, beta=beta, include_llist=False, line_margin=0.3)
    c1, _ = opacity(comps, lam, nu, cells, beta=beta, include_llist=True, line_margin=0.3)
    assert np.all(c1 >= c0 * (1 - 2e-7)) and np.mean(c1 > c0 * 1.001) > 0.05


def test_opacity_full_case_beta_from_nu(m3d, oracle):
    from oracle import continuum as oc
    from dispatch_b200.continuum import opacity
    atm, lam, nu, llam, comps, cells = _case()
    m3d.hop_set_state(atm)
    chi, scat = opacity(comps, lam, nu, cells, line_margin=0.3)
    hk = 6.626176e-27 / 1.380662e-16
    beta = np.maximum(np.exp(-nu[None, :] * (hk / cells["temp"][:, None])).astype(np.float32),
                      np.float32(np.finfo(np.float32).tiny))
    want, so = _oracle(oracle, oc, atm, lam, nu, llam, comps, cells, beta, 0.3)
    assert np.all(np.isfinite(chi)) and np.all(chi > 0)
    np.testing.assert_allclose(scat, so, rtol=1e-6)
    np.testing.assert_allclose(chi, want, rtol=1e-5)
    with pytest.raises(m3d.M3DError, match="uniform in ln"):
        opacity(comps, np.linspace(lam[0], lam[-1] * 1.01, lam.size), nu, cells)


def test_chi500(m3d):
    """load_state_variables' chi500: the pipeline at one wavelength without the line
    list, needing no loaded state; equal to the continuum's xhat (1 - beta) + sigma."""
    from dispatch_b200.continuum import air2vac, chi500, continuum_opacities
    m3d.lib().m3d_hop_free_state()   # chi500 needs no line list
    comps, _, _, cells = synth.continuum_case(ncell=700, nlam=8)
    c5 = chi500(comps, cells)
    assert c5.shape == (700,) and np.all(np.isfinite(c5)) and np.all(c5 > 0)
    lam = np.atleast_1d(air2vac(5000.0))
    assert 5001.0 < lam[0] < 5002.0              # 5000 A air is 5001.40 A vacuum
    nu = (2.99792458e10 / 1e-8) / lam
    xh, sg = continuum_opacities(comps, lam, nu, cells)
    hk = 6.626176e-27 / 1.380662e-16
    beta = np.maximum(np.exp(-nu[0] * (hk / cells["temp"])), np.finfo(np.float32).tiny).astype(np.float32)
    np.testing.assert_allclose(c5, xh[:, 0] * (np.float32(1) - beta) + sg[:, 0], rtol=1e-5)

"""m3d_hop_opacity: hop_opacity's argument list (libhop.h:20) on this library's line
opacity.  On a loaded state and a continuum filled in by the caller, the line list
is added as add_linelist_opacities adds it -- an accumulator from zero against the
continuum as the tolerance reference, the lines within line_margin -- bit for bit
against the oracle's add_opacity_equi on the same inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_hop_opacity_matches_oracle(m3d, oracle):
    from dispatch_b200 import synth
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=48, window=3)
    ncell = atm["temp"].size
    lam = np.exp(llam)
    beta, Bnu = oracle.lte_background(nu, atm["temp"])
    cont, _ = oracle.lte_work(atm["chi_c"], beta, Bnu)           # the caller's continuum (ncell, nlam)
    cont = np.ascontiguousarray(cont, np.float32)
    chi = cont.copy()
    scat = np.zeros_like(chi)
    m3d.hop_set_state(atm)
    margin = 0.3
    m3d.hop_opacity(lam, chi, scat, 0, 1, margin, -1)
    # the oracle: the same selection, a zero accumulator, then added to the continuum
    sp = dict(atm["species"][0])
    lo, hi = llam[0] - margin / lam[0], llam[-1] + margin / lam[0]
    sp["active"] = ((sp["llam0"] >= lo) & (sp["llam0"] <= hi)).astype(np.uint8)
    assert 0 < sp["active"].sum() < sp["active"].size
    chil = np.zeros_like(chi)
    etal = np.zeros_like(chi)
    cells = {"vproj": np.zeros(ncell, np.float32), "inv_df": sp["inv_df"], "vbar2": sp["vbar2"],
             "lnbase": sp["lnbase"], "e_kT": atm["e_kT"], "ne": atm["ne"], "tothi": atm["tothi"],
             "stark_pe": atm["stark_pe"]}
    oracle.add_opacity_equi(sp, llam, chil, etal, cont, oracle.logref(cont), cells)
    np.testing.assert_array_equal(chi, (cont + chil).astype(np.float32))
    assert np.all(scat == 0)
    # what it leaves to the caller
    with pytest.raises(m3d.M3DError, match="include_absmet"):
        m3d.hop_opacity(lam, chi, scat, 1, 1, margin, -1)
    with pytest.raises(m3d.M3DError, match="uniform in ln"):
        m3d.hop_opacity(np.linspace(lam[0], lam[-1] * 1.01, lam.size), chi, scat, 0, 1, margin, -1)

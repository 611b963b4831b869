"""GPU parity of the model-atom opacity and rate kernels against the oracle.

Every comparison is bit-exact: the kernels and the restatement perform the
same IEEE operations in the same order per point (transitions in window order
at each (f, cell), frequencies in order for each (transition, cell) sum); the
one libm call on these paths, the power of a van der Waals recipe that is
not Unsold's, is compared with a relative tolerance of 1e-6.
"""
import numpy as np
import pytest

from tests import nlte_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nl(oracle):
    from oracle import nlte
    return nlte


@pytest.fixture(scope="module")
def gn(m3d):
    from dispatch_b200 import nlte
    return nlte


@pytest.fixture(scope="module")
def base():
    return nlte_cases.case(ncell=300, sums_every=7)


def _split(n, nf):
    z = lambda dt: np.zeros((n, nf), dt)
    return {"opac_L": z(np.float32), "opac_R": z(np.float32), "id": z(np.int32),
            "chi_L": z(np.float32), "chi_R": z(np.float32), "chi_id": z(np.int32)}


def test_damping(nl, gn, base):
    atom, inp, win, c, field = base
    args = [c[k] for k in ("ne", "tothi", "vbar2", "stark_pe", "unsold", "inv_df")]
    assert np.array_equal(gn.bb_damping(win, *args), nl.bb_damping(win, *args))
    w2 = dict(win)
    L = win["nline"]
    w2["gw1"] = np.where(np.arange(L) % 3 == 0, 1e-8, 0.0)
    w2["gw2"] = np.full(L, 0.4)
    w2["unsold"] = (np.arange(L) % 3 == 1).astype(np.uint8)
    w2["gstk"] = np.where(np.arange(L) % 2 == 0, 1e-15, -2e-15)
    np.testing.assert_allclose(gn.bb_damping(w2, *args), nl.bb_damping(w2, *args), rtol=1e-6)


@pytest.mark.parametrize("lte", [False, True])
def test_opacities_and_split(nl, gn, base, lte):
    atom, inp, win, c, field = base
    n, nf = c["pop_ratio"].size, win["nf"]
    adamp = nl.bb_damping(win, c["ne"], c["tothi"], c["vbar2"], c["stark_pe"], c["unsold"], c["inv_df"])
    res = []
    for mod in (nl, gn):
        xh, eh = field["xhat"].copy(), field["ehat"].copy()
        mod.bf_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], xh, eh)
        sp = _split(n, nf)
        wphi = np.zeros((atom["nline"], n), np.float32)
        mod.bb_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, xh, eh,
                       lte=lte, wmu=0.3, split=sp, wphi=wphi)
        res.append((xh, eh, sp, wphi))
    (xo, eo, so, wo), (xg, eg, sg, wg) = res
    assert np.array_equal(xg, xo) and np.array_equal(eg, eo)
    for k in so:
        assert np.array_equal(sg[k], so[k]), k
    assert np.array_equal(wg, wo) and np.count_nonzero(wg) > 0


def test_bf_opacity_cut_and_lte(nl, gn):
    atom, inp, win, c, field = nlte_cases.case(ncell=120, cut_x=12.0)
    for b in (c["b"], None):
        r = []
        for mod in (nl, gn):
            xh, eh = field["xhat"].copy(), field["ehat"].copy()
            mod.bf_opacity(win, b, c["nstar"], c["pop_ratio"], c["e_kT"], xh, eh)
            r.append((xh, eh))
        assert np.array_equal(r[0][0], r[1][0]) and np.array_equal(r[0][1], r[1][1])


def test_transfer_units_split(nl, gn, base):
    atom, inp, win, c, field = base
    n, nf = c["pop_ratio"].size, win["nf"]
    adamp = nl.bb_damping(win, c["ne"], c["tothi"], c["vbar2"], c["stark_pe"], c["unsold"], c["inv_df"])
    xh, eh = field["xhat"].copy(), field["ehat"].copy()
    sp = _split(n, nf)
    nl.bb_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, xh, eh, split=sp)
    scat = (0.01 * field["Bnu"]).astype(np.float32)
    for sc in (None, scat):
        for sup in (False, True):
            r = []
            for mod in (nl, gn):
                w1, w2 = xh.copy(), eh.copy()
                nfl = mod.transfer_units_split(w1, w2, field["beta"], sp, scat=sc, suppress_masers=sup)
                r.append((w1, w2, nfl))
            assert np.array_equal(r[0][0], r[1][0]) and np.array_equal(r[0][1], r[1][1]) and r[0][2] == r[1][2]


def test_bb_opacity_units_fused(nl, gn, base):
    """m3d_bb_opacity_units: the opacity and the split transfer units in one pass from
    the background, against the oracle's bb_opacity then transfer_units_split on a
    copy of it."""
    atom, inp, win, c, field = base
    n, nf = c["pop_ratio"].size, win["nf"]
    adamp = nl.bb_damping(win, c["ne"], c["tothi"], c["vbar2"], c["stark_pe"], c["unsold"], c["inv_df"])
    xh, eh = field["xhat"].copy(), field["ehat"].copy()
    nl.bf_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], xh, eh)
    w1, w2 = xh.copy(), eh.copy()
    so = _split(n, nf)
    wo = np.zeros((atom["nline"], n), np.float32)
    nl.bb_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, w1, w2,
                  wmu=0.3, split=so, wphi=wo)
    nl.transfer_units_split(w1, w2, field["beta"], so)
    chi, S = np.zeros_like(w1), np.zeros_like(w2)
    sg = _split(n, nf)
    wg = np.zeros((atom["nline"], n), np.float32)
    gn.bb_opacity_units(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, xh, eh,
                        field["beta"], chi, S, sg, wmu=0.3, wphi=wg)
    assert np.array_equal(chi, w1) and np.array_equal(S, w2)
    for k in so:
        assert np.array_equal(sg[k], so[k]), k
    assert np.array_equal(wg, wo)


@pytest.mark.parametrize("split_rates,precond", [(True, True), (True, False), (False, True), (False, False)])
def test_bb_rates(nl, gn, base, split_rates, precond):
    atom, inp, win, c, field = base
    n, nf = c["pop_ratio"].size, win["nf"]
    ntr = win["nline"] + win["ncont"]
    adamp = nl.bb_damping(win, c["ne"], c["tothi"], c["vbar2"], c["stark_pe"], c["unsold"], c["inv_df"])
    xh, eh = field["xhat"].copy(), field["ehat"].copy()
    sp = _split(n, nf)
    nl.bb_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, xh, eh, split=sp)
    w1, w2 = xh.copy(), eh.copy()
    nl.transfer_units_split(w1, w2, field["beta"], sp)
    nwords = (atom["nline"] + 31) // 32 + 1
    rng = np.random.default_rng(5)
    fin = (rng.random((nwords, n)) < 0.5).astype(np.uint32) * rng.integers(0, 2**32, (nwords, n), dtype=np.uint32)
    scat = (0.01 * field["Bnu"]).astype(np.float32)
    out = []
    for mod in (nl, gn):
        gij = (0.1 * np.ones((ntr, n))).astype(np.float32)
        gji = np.zeros((ntr, n), np.float32)
        fr = np.zeros((nwords, n), np.uint32)
        mod.bb_rates(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp,
                     field["inu"], field["beta"], field["Bnu"], gij, gji, work1=w1, psi=field["psi"],
                     irem=field["irem"], escape=field["escape"], split=sp, scat=scat if split_rates else None,
                     flags_in=fin if split_rates else None, flags_raise=fr if split_rates else None,
                     split_rates=split_rates, preconditioning=precond, wmu=0.25, wtot=1.0)
        out.append((gij, gji, fr))
    (go, jo, fo), (gg, jg, fg) = out
    assert np.array_equal(gg, go) and np.array_equal(jg, jo) and np.array_equal(fg, fo)
    if split_rates and precond:
        assert np.count_nonzero(fg) > 0


def test_bf_rates_integrate_normalize(nl, gn, base):
    atom, inp, win, c, field = base
    n, nf = c["pop_ratio"].size, win["nf"]
    ntr = win["nline"] + win["ncont"]
    J = field["inu"]
    for precond in (True, False):
        r = []
        for mod in (nl, gn):
            gij = np.zeros((ntr, n), np.float32)
            gji = np.zeros((ntr, n), np.float32)
            mod.bf_rates(win, c["b"], c["nstar"], c["e_kT"], J, field["psi"], field["beta"], gij, gji,
                         preconditioning=precond)
            r.append((gij, gji))
        assert np.array_equal(r[0][0], r[1][0]) and np.array_equal(r[0][1], r[1][1])
    gw_ij, gw_ji = r[1]
    gw_ij[: win["nline"]] = 1.5
    gw_ji[: win["nline"]] = 0.5
    nrad = len(atom["ti"])
    gi, gj = np.ones((nrad, n), np.float32), np.ones((nrad, n), np.float32)
    gn.integrate_rates(win, gw_ij, gw_ji, gi, gj)
    assert np.array_equal(gi, 1 + gw_ij) and np.array_equal(gj, 1 + gw_ji)
    has = (np.arange(atom["nline"]) % 7 == 0).astype(np.uint8)
    wphi = np.random.default_rng(2).random((atom["nline"], n)).astype(np.float32)
    wphi[0, :5] = 0
    for first in (True, False):
        r = []
        for mod in (nl, gn):
            a, b, w = gi.copy(), gj.copy(), wphi.copy()
            mod.normalize_profiles(atom, c["nstar"], w, a, b, has, first)
            r.append((a, b, w))
        for x, y in zip(*r):
            assert np.array_equal(x, y)


def test_combine_twins(gn):
    rng = np.random.default_rng(0)
    a = rng.random(1000).astype(np.float32)
    b = rng.random(1000).astype(np.float32)
    ref = (np.float32(0.5) * (a + b)).astype(np.float32)
    gn.combine_twins(a, b)
    assert np.array_equal(a, ref) and np.array_equal(b, ref)

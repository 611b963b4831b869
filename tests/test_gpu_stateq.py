"""GPU parity of the statistical-equilibrium kernels against the oracle.

Bit-exact where both sides perform the same IEEE operations in the same
order: the rate matrix, the three dense solves and the update of every cell
(with the collision rates taken from the oracle and no correction at the
limiter).  The collision recipes, the limiter's exp/pow and Ng's log/exp call
the device's double-precision exp and log, which may differ from the host's
by an ulp: rates compared directly carry a relative tolerance of 1e-12, and
populations solved from them 1e-10, the ulp differences amplified by the rate
matrix's conditioning (stated per test); the reference's own requirement on
departure coefficients is 1e-4.
"""
import numpy as np
import pytest

from dispatch_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sq(oracle):
    from oracle import stateq
    return stateq


@pytest.fixture(scope="module")
def se(m3d):
    from dispatch_b200 import stateq
    return stateq


def _oracle_update(sq, atom, inp, cup, **kw):
    b = inp["b"].copy()
    res, lvlerr, rc = sq.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                       inp["gamma_ji"], temp=inp["temp"], cup=cup, **kw)
    return b, res, lvlerr, rc


def _gpu_update(se, atom, inp, cup=None, **kw):
    b = inp["b"].copy()
    res, lvlerr = se.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                   inp["gamma_ji"], temp=inp["temp"], ne=inp["ne"], cup=cup, **kw)
    res.pop("team")
    return b, res, lvlerr


def test_collision_rates(sq, se):
    for nb, nl in ((20, 60), (60, 180)):
        atom, inp = synth.se_config("small", ncell=1024, nbound=nb, nline=nl)
        ref = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
        got = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
        assert np.all(np.isfinite(got)) and np.count_nonzero(got) > 0.9 * got.size
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)   # device exp/log
        dxi = np.full_like(inp["temp"], 0.05)
        ref = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], dxi)
        got = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], dxi)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("solver", [0, 1, 2])
@pytest.mark.parametrize("nbound,nline", [(20, 60), (60, 180)])
def test_update_bitexact(sq, se, solver, nbound, nline):
    atom, inp = synth.se_config("small", ncell=1500, nbound=nbound, nline=nline)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup, solver=solver)
    assert rc == 0 and ro["nclamp"] == 0
    bg, rg, lg = _gpu_update(se, atom, inp, cup=cup, solver=solver)
    assert np.array_equal(bg, bo)
    assert rg == ro
    assert np.array_equal(lg, lo)


@pytest.mark.parametrize("nbound,nline", [(20, 60), (60, 180)])
@pytest.mark.parametrize("form", ["cup", "fused", "hydrogen", "gencol"])
def test_update_team_equals_warp(se, nbound, nline, form):
    """A cell solved by a block of 64 or 128 threads (the library's choice for a
    large atom under lineq_no_pivot) gives the bits of one warp per cell, with the
    collision rates read, formed from the electron recipes, with the hydrogen
    recipes, and with tabulated records."""
    kw = {}
    if form == "hydrogen":
        kw["h_recipes"] = H_RECIPES
    if form == "gencol":
        kw["gencol"] = True
    atom, inp = synth.se_config("small", ncell=3000, nbound=nbound, nline=nline, **kw)
    cup = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"]) if form == "cup" else None
    cell_kw = _cell_kw(inp) if form in ("hydrogen", "gencol") else {}
    out = []
    for warp in (False, True):
        b = inp["b"].copy()
        res, lvlerr = se.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                       inp["gamma_ji"], temp=inp["temp"], ne=inp["ne"], cup=cup,
                                       warp_per_cell=warp, **cell_kw)
        out.append((b, res, lvlerr))
    assert out[1][1]["team"] == 32
    if nbound == 60:
        assert out[0][1]["team"] > 32
    for k in ("team",):
        out[0][1].pop(k)
        out[1][1].pop(k)
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    assert out[0][1]["maxerr"] != 0


def test_update_rounds_inactive_cut(sq, se):
    """A pair carrying two lines (two rounds of additions), inactive
    transitions, and the radiative cut's detailed-balance pair (cut_x = 20)."""
    atom, inp = synth.se_config("small", ncell=800)
    atom = dict(atom)
    nl = atom["nline"]
    # duplicate line 3 as an extra line of the same pair; the continua keep their order
    ti = np.concatenate([atom["ti"][:nl], [atom["ti"][3]], atom["ti"][nl:]]).astype(np.int32)
    tj = np.concatenate([atom["tj"][:nl], [atom["tj"][3]], atom["tj"][nl:]]).astype(np.int32)
    aji = np.concatenate([atom["Aji"][:nl], [0.5 * atom["Aji"][3]], atom["Aji"][nl:]])
    act = np.ones(len(ti), np.uint8)
    act[[7, 30, nl + 1 + 4]] = 0
    atom.update(ti=ti, tj=tj, Aji=aji, nline=nl + 1, active=act, cut_x=20.0)
    inp = dict(inp)
    for k in ("gamma_ij", "gamma_ji"):
        g = inp[k]
        inp[k] = np.ascontiguousarray(np.concatenate([g[:nl], 0.7 * g[3:4], g[nl:]]))
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup)
    assert rc == 0
    bg, rg, lg = _gpu_update(se, atom, inp, cup=cup)
    assert np.array_equal(bg, bo) and rg == ro and np.array_equal(lg, lo)


def test_update_fused_collisions(sq, se):
    atom, inp = synth.se_config("small", ncell=2048)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup)
    bg, rg, lg = _gpu_update(se, atom, inp, cup=None)
    # the collision rates agree to 1e-12 (device exp/log); the solve amplifies that
    # by the rate matrix's conditioning
    np.testing.assert_allclose(bg, bo, rtol=1e-10, atol=0)
    assert rg["epos_cell"] == ro["epos_cell"] and rg["epos_level"] == ro["epos_level"]
    assert rg["maxerr"] == pytest.approx(ro["maxerr"], rel=1e-10)


H_RECIPES = ("drawin", "drawin", "takeda")


def test_collision_rates_hydrogen(sq, se):
    """Drawin and Takeda (atom_mod.f90:1854-1876) beside the electron recipes."""
    atom, inp = synth.se_config("small", ncell=1024, h_recipes=H_RECIPES)
    ncol = len(atom["col_i"])
    dxi = np.full_like(inp["temp"], 0.05)
    ref = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], dxi, nh1=inp["nh1"])
    got = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], dxi, nh1=inp["nh1"])
    assert got.shape == ref.shape == (2 * ncol, 1024)
    assert np.count_nonzero(got[ncol:]) > 0.9 * ncol * 1024
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)   # device exp


@pytest.mark.parametrize("solver", [0, 1, 2])
def test_update_bitexact_hydrogen(sq, se, solver):
    atom, inp = synth.se_config("small", ncell=1500, h_recipes=H_RECIPES)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup, solver=solver)
    assert rc == 0
    bg, rg, lg = _gpu_update(se, atom, inp, cup=cup, solver=solver)
    assert np.array_equal(bg, bo) and rg == ro and np.array_equal(lg, lo)
    # the hydrogen rates move the solution
    b0, _, _, _ = _oracle_update(sq, dict(atom, col_hkind=None), inp, cup[:len(atom["col_i"])], solver=solver)
    assert not np.array_equal(b0, bo)


def test_update_fused_hydrogen(sq, se):
    atom, inp = synth.se_config("small", ncell=2048, h_recipes=H_RECIPES)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup)
    bg, rg, lg = _gpu_update(se, atom, inp, cup=None, nh1=inp["nh1"])
    # the rates agree to 1e-12 (device exp); the solve amplifies that by the rate
    # matrix's conditioning, here up to 1.2e-10
    np.testing.assert_allclose(bg, bo, rtol=5e-10, atol=0)
    assert rg["epos_cell"] == ro["epos_cell"] and rg["epos_level"] == ro["epos_level"]
    # forming the rates inside the update equals passing the device's own rates
    cupd = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    bd, rd, ld = _gpu_update(se, atom, inp, cup=cupd)
    assert np.array_equal(bg, bd) and rg == rd and np.array_equal(lg, ld)


def test_hydrogen_recipe_checks(se):
    from dispatch_b200 import M3DError
    atom, inp = synth.se_config("small", ncell=64, h_recipes=H_RECIPES)
    args = (inp["temp"], inp["ne"], inp["e_kT"])
    with pytest.raises(M3DError, match="nh1"):
        se.collision_rates(atom, *args)
    hk = atom["col_hkind"].copy()
    bad = dict(atom, col_hkind=np.where(atom["col_fac"] != 0, 2, hk).astype(np.int32))
    with pytest.raises(M3DError, match="Takeda"):
        se.collision_rates(bad, *args, nh1=inp["nh1"])
    hk[0] = 7
    with pytest.raises(M3DError, match="hydrogen kind"):
        se.collision_rates(dict(atom, col_hkind=hk), *args, nh1=inp["nh1"])
    b = inp["b"].copy()
    with pytest.raises(M3DError, match="nh1"):
        se.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"], inp["gamma_ji"],
                         temp=inp["temp"], ne=inp["ne"])
    assert np.array_equal(b, inp["b"])


def _gencol_case(ncell):
    return synth.se_config("small", ncell=ncell, gencol=True, h_recipes=H_RECIPES)


def _cell_kw(inp):
    return {k: inp[k] for k in ("nh1", "lsaha", "colliders")}


def test_collision_rates_gencol(sq, se):
    """gencol's records (atom_mod.f90:2223-2360), the Saha branch where n*_ll = 0."""
    atom, inp = _gencol_case(1024)
    nstar = inp["nstar"].copy()
    nstar[atom["gencol"]["ll"], :64] = 0.0
    dxi = np.full_like(inp["temp"], 0.05)
    ref = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], dxi, nstar=nstar, **_cell_kw(inp))
    got = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], dxi, nstar=nstar, **_cell_kw(inp))
    assert got.shape == ref.shape == (se.collision_nrows(atom), 1024)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)   # device exp/log
    # the library's node slopes are the oracle's
    gc = dict(atom["gencol"], dlnc=sq.hermite_derivative(atom["gencol"]["tgrid"], atom["gencol"]["lnc"]))
    got2 = se.collision_rates(dict(atom, gencol=gc), inp["temp"], inp["ne"], inp["e_kT"], dxi, nstar=nstar,
                              **_cell_kw(inp))
    assert np.array_equal(got2, got)


@pytest.mark.parametrize("solver", [0, 1, 2])
def test_update_bitexact_gencol(sq, se, solver):
    atom, inp = _gencol_case(1500)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nstar=inp["nstar"], **_cell_kw(inp))
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup, solver=solver)
    assert rc == 0
    bg, rg, lg = _gpu_update(se, atom, inp, cup=cup, solver=solver)
    assert np.array_equal(bg, bo) and rg == ro and np.array_equal(lg, lo)


def test_update_fused_gencol(sq, se):
    atom, inp = _gencol_case(2048)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nstar=inp["nstar"], **_cell_kw(inp))
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup)
    bg, rg, lg = _gpu_update(se, atom, inp, cup=None, **_cell_kw(inp))
    np.testing.assert_allclose(bg, bo, rtol=5e-10, atol=0)   # device exp/log, amplified by the solve
    assert rg["epos_cell"] == ro["epos_cell"] and rg["epos_level"] == ro["epos_level"]
    cupd = se.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nstar=inp["nstar"], **_cell_kw(inp))
    bd, rd, ld = _gpu_update(se, atom, inp, cup=cupd)
    assert np.array_equal(bg, bd) and rg == rd and np.array_equal(lg, ld)


def test_gencol_checks(se):
    from dispatch_b200 import M3DError
    atom, inp = _gencol_case(64)
    args = (inp["temp"], inp["ne"], inp["e_kT"])
    kw = _cell_kw(inp)
    with pytest.raises(M3DError, match="nstar"):
        se.collision_rates(atom, *args, **kw)
    with pytest.raises(M3DError, match="lsaha"):
        se.collision_rates(atom, *args, nstar=inp["nstar"], nh1=inp["nh1"], colliders=inp["colliders"])
    with pytest.raises(M3DError, match="ncollider"):
        se.collision_rates(atom, *args, nstar=inp["nstar"], nh1=inp["nh1"], lsaha=inp["lsaha"],
                           colliders=inp["colliders"][:1])
    gc = dict(atom["gencol"], collider=np.full(len(atom["gencol"]["ll"]), -1, np.int32))
    with pytest.raises(M3DError, match="collider row"):
        se.collision_rates(dict(atom, gencol=gc), *args, nstar=inp["nstar"], **kw)
    gc = dict(atom["gencol"], tgrid=atom["gencol"]["tgrid"][::-1].copy())
    with pytest.raises(M3DError, match="ascending"):
        se.collision_rates(dict(atom, gencol=gc), *args, nstar=inp["nstar"], **kw)


def test_update_limiter_sor_floor(sq, se):
    atom, inp = synth.se_config("small", ncell=1024)
    inp = dict(inp)
    b = inp["b"].copy()
    b[3, :40] *= 1e-6
    b[5, 40:60] *= 1e5
    inp["b"] = b
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    kw = dict(sor_w=0.7, conv_pop_floor=1e-3, min_pop_frac=1e-12)
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup, **kw)
    assert rc == 0 and ro["nclamp"] >= 60
    bg, rg, lg = _gpu_update(se, atom, inp, cup=cup, **kw)
    np.testing.assert_allclose(bg, bo, rtol=1e-10, atol=0)   # limiter exp, e**sor_w, amplified by the solve
    assert rg["nclamp"] == ro["nclamp"] and rg["ntot"] == ro["ntot"]
    assert (rg["epos_cell"], rg["epos_level"]) == (ro["epos_cell"], ro["epos_level"])
    np.testing.assert_allclose(lg, lo, rtol=1e-10)


def test_update_skips_and_nonfinite(sq, se):
    atom, inp = synth.se_config("small", ncell=256)
    inp = dict(inp)
    totn = inp["totn"].copy()
    totn[10] = 0.0
    temp = inp["temp"].copy()
    temp[11] = 2e7
    g = inp["gamma_ij"].copy()
    g[0, 5] = np.nan
    g[2, 200] = np.inf
    inp.update(totn=totn, temp=temp, gamma_ij=g)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    bo, ro, lo, rc = _oracle_update(sq, atom, inp, cup)
    assert rc == 5 and ro["nonfinite_cell"] == 5
    b = inp["b"].copy()
    with pytest.raises(se.NonFiniteSolution) as ei:
        se.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"], inp["gamma_ji"],
                         temp=inp["temp"], cup=cup)
    ei.value.result.pop("team")
    assert ei.value.result == ro
    for c in (5, 10, 11, 200):
        assert np.array_equal(b[:, c], inp["b"][:, c])
    assert np.array_equal(b, bo)


def test_update_device_pointers(sq, se):
    torch = pytest.importorskip("torch")
    atom, inp = synth.se_config("small", ncell=777)
    bh, rh, lh = _gpu_update(se, atom, inp)
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in inp.items()}
    rd, ld = se.stateq_update(atom, d["b"], d["nstar"], d["totn"], d["e_kT"], d["gamma_ij"], d["gamma_ji"],
                              temp=d["temp"], ne=d["ne"])
    rd.pop("team")
    assert np.array_equal(d["b"].cpu().numpy(), bh) and rd == rh and np.array_equal(ld, lh)


def _ng_case(seed=3, nlevel=21, ncell=5000):
    rng = np.random.default_rng(seed)
    xinf = rng.normal(0, 0.5, (nlevel, ncell))
    v1, v2, v3 = rng.normal(0, 0.1, (3, nlevel, ncell))
    it = [np.exp(xinf + 0.8**k * v1 + 0.5**k * v2 + 0.3**k * v3) for k in range(4)]
    nstar = np.exp(rng.normal(0, 2, (nlevel, ncell)))
    totn = (np.exp(xinf) * nstar).sum(axis=0)
    return np.ascontiguousarray(np.stack(it[:3])), np.ascontiguousarray(it[3]), nstar, totn


def test_ng_accumulate_extrapolate(sq, se):
    oldb, b, nstar, totn = _ng_case()
    go = sq.ng_accumulate(b, oldb)
    gg = se.ng_accumulate(b, oldb)
    np.testing.assert_allclose(gg, go, rtol=1e-11)   # summation order differs (tree vs sequential)
    st = se.NgState()
    st.d_done = go[:6].copy()
    st.coefficients()
    bo, bg = b.copy(), b.copy()
    ro = sq.ng_extrapolate(bo, oldb, nstar, totn, st.a, st.b)
    rg = se.ng_extrapolate(bg, oldb, nstar, totn, st.a, st.b)
    assert ro["applied"] and rg["applied"]
    np.testing.assert_allclose(bg, bo, rtol=1e-12)   # device log/exp
    assert (rg["epos_cell"], rg["epos_level"]) == (ro["epos_cell"], ro["epos_level"])
    assert rg["emax"] == pytest.approx(ro["emax"], rel=1e-9)
    # the veto leaves b as it was
    bv = b.copy()
    rv = se.ng_extrapolate(bv, oldb, nstar, totn, st.a, st.b, max_change=1e-9)
    assert not rv["applied"] and np.array_equal(bv, b) and rv["epos_cell"] == -1
    rv = se.ng_extrapolate(bv, oldb, nstar, totn, float("nan"), st.b)
    assert not rv["applied"] and np.array_equal(bv, b)


def test_ng_driver_fires_on_geometric_sequence(se):
    """The whole host gate over a slowly contracting two-mode sequence: Ng
    waits for a stationary rate, fires, and lands on the limit."""
    rng = np.random.default_rng(9)
    nlevel, ncell = 8, 3000
    xinf = rng.normal(0, 0.4, (nlevel, ncell))
    v1, v2 = rng.normal(0, 0.2, (2, nlevel, ncell))
    nstar = np.ones((nlevel, ncell))
    totn = np.exp(xinf).sum(axis=0)
    st = se.NgState()
    oldb = np.ascontiguousarray(np.stack([np.exp(xinf + v1 + v2)] * 3))
    fired = None
    for it in range(1, 16):
        b = np.ascontiguousarray(np.exp(xinf + 0.9**it * v1 + 0.6**it * v2))
        err = float(np.max(np.abs(b / oldb[2] - 1)))
        if it >= 2:
            st.count_clamped(0, b.size)
        out = se.ng_acceleration(st, it, err, 1e-8, b, oldb if it >= 3 else None, nstar, totn)
        if out["applied"]:
            fired = it
            break
        se.shift_oldb(oldb, b)
    assert fired is not None
    assert np.max(np.abs(np.log(b) - xinf)) < 1e-6


def test_c2_full_size(sq, se):
    """The 120^3 cube of the 3D NLTE configuration with its 21-level atom:
    LTE gives b = 1 in every cell; the non-LTE update conserves particles."""
    atom, inp = synth.se_config("c2", lte=True)
    b, res, lvl = _gpu_update(se, atom, inp)
    assert res["nonfinite_cell"] == -1 and res["ntot"] == inp["totn"].size * atom["nlevel"]
    assert np.max(np.abs(b - 1.0)) < 2e-6
    atom, inp = synth.se_config("c2")
    b, res, lvl = _gpu_update(se, atom, inp)
    assert np.all(np.isfinite(b)) and np.all(b > 0)
    np.testing.assert_allclose((b * inp["nstar"]).sum(axis=0), inp["totn"], rtol=1e-12)
    # a sample of cells against the oracle
    idx = np.arange(0, inp["totn"].size, 7919)
    sub = {k: np.ascontiguousarray(v[..., idx]) for k, v in inp.items()}
    cup = sq.collision_rates(atom, sub["temp"], sub["ne"], sub["e_kT"])
    bo = _oracle_update(sq, atom, sub, cup)[0]
    np.testing.assert_allclose(b[:, idx], bo, rtol=1e-10)

"""gencol, the atom file's tabulated collision records, in the SE oracle (CPU only).

  * hermite_derivative's interior slopes are the Fritsch-Butland harmonic means of
    scipy's PchipInterpolator, its end slopes the quadratic 2 dy/dx - d of the
    neighbour (interpol_mod.f90:240-284); hermite_interpolation (:558-578) is the
    cubic Hermite spline on those slopes, clamped to the end values outside;
  * each record kind's upward and downward rates worked by hand for one cell
    (atom_mod.f90:2288-2344), with the Saha branch of n_ul/n_ll where n*_ll = 0;
  * the rate matrix adds the records after classic_col's rates into the same
    matrix elements (collision_rates :918-930, setup_transition_matrix :806-811);
  * the records keep detailed balance: LTE still gives b = 1.
"""
import math

import numpy as np
import pytest

from dispatch_b200 import stateq, synth

H_RECIPES = ("drawin", "drawin", "takeda")


@pytest.fixture(scope="module")
def sq(oracle):
    from oracle import stateq as s
    return s


def _case(ncell=64, **kw):
    return synth.se_config("small", ncell=ncell, gencol=True, h_recipes=H_RECIPES, **kw)


def _rates(sq, atom, inp, nstar=None):
    return sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"],
                              nstar=inp["nstar"] if nstar is None else nstar, lsaha=inp["lsaha"],
                              colliders=inp["colliders"])


def test_hermite_slopes_and_interpolation(sq):
    interpolate = pytest.importorskip("scipy.interpolate")
    rng = np.random.default_rng(4)
    x = np.sort(rng.uniform(1.0, 10.0, 12))
    for y in (np.cumsum(rng.uniform(0.1, 1.0, 12)), np.sin(x), -np.log(x)):
        d = sq.hermite_derivative(x, y[None, :])[0]
        ref = interpolate.PchipInterpolator(x, y).derivative()(x)
        np.testing.assert_allclose(d[1:-1], ref[1:-1], rtol=1e-12, atol=1e-14)
        assert d[0] == 2.0 * (y[1] - y[0]) / (x[1] - x[0]) - d[1]
        assert d[-1] == 2.0 * (y[-1] - y[-2]) / (x[-1] - x[-2]) - d[-2]
        spline = interpolate.CubicHermiteSpline(x, y, d)
        for xx in np.concatenate([rng.uniform(x[0], x[-1], 40), x[1:-1]]):
            assert sq.hermite_interp(x, y, d, xx) == pytest.approx(float(spline(xx)), rel=1e-12, abs=1e-13)
        assert sq.hermite_interp(x, y, d, x[0] - 1.0) == y[0]
        assert sq.hermite_interp(x, y, d, x[-1] + 1.0) == y[-1]
    # a flat stretch and a sign change give zero interior slopes
    y = np.array([0.0, 1.0, 1.0, 2.0, 1.0])
    d = sq.hermite_derivative(np.arange(5.0), y[None, :])[0]
    assert d[1] == 0 and d[2] == 0 and d[3] == 0
    d2 = sq.hermite_derivative(np.array([1.0, 3.0]), np.array([[2.0, 6.0]]))[0]
    assert d2[0] == d2[1] == 2.0


def _by_hand(sq, atom, inp, c, r, nll, nul):
    gc = atom["gencol"]
    ll, ul, kind = int(gc["ll"][r]), int(gc["ul"][r]), int(gc["kind"][r])
    ev, g, ion = atom["ev"], atom["g"], atom["ion"]
    T, ne, ekt, nh1, ls = inp["temp"][c], inp["ne"][c], inp["e_kT"][c], inp["nh1"][c], inp["lsaha"][c]
    dev = ev[ul] - ev[ll]
    nji = nul / nll if nll > 0 else g[ul] / g[ll] * math.exp(-dev * ekt + (ion[ul] - ion[ll]) * ls)
    x = gc["tgrid"]
    d = sq.hermite_derivative(x, gc["lnc"][r:r + 1])[0]
    ct = math.exp(sq.hermite_interp(x, gc["lnc"][r], d, T))
    stg = math.sqrt(T)
    eryd = 13.605 * 1.602189e-12
    c0 = ((eryd / math.sqrt(9.109534e-28)) * 3.14159265359 * 5.29177349e-9**2) * math.sqrt(
        8.0 / (3.14159265359 * 1.380662e-16))
    col = gc["collider"][r]
    ncoll = inp["colliders"][col, c] if col >= 0 else 0.0
    if kind == 1:
        dn = c0 / g[ul] * ct * ne / stg
        up = dn * nji
    elif kind == 2:
        dn = g[ll] / g[ul] * ct * ne * stg
        up = dn * nji
    elif kind == 3:
        dn = ct * nh1
        up = dn * nji
    elif kind == 4:
        up = ct * nh1
        dn = up / nji
    elif kind == 5:
        up = ct * ne * stg * math.exp(-dev * ekt)
        dn = up / nji
    elif kind == 6:
        up = ct * nh1 * (math.exp(-float(np.float32(0.754)) * ekt) if gc["ch0_hmip"] else 1.0)
        dn = up / nji
    elif kind == 7:
        up = ct * ncoll
        dn = up / nji
    elif kind == 8:
        dn = ct * ncoll
        up = dn * nji
    else:
        up = dn = 0.0
    return up, dn


def test_record_rates_by_hand(sq):
    atom, inp = _case(ncell=16)
    cup = _rates(sq, atom, inp)
    gc = atom["gencol"]
    nrec = len(gc["ll"])
    r0 = stateq.collision_nrows(atom) - 2 * nrec
    assert r0 == 2 * len(atom["col_i"]) and np.all(np.isfinite(cup)) and np.all(cup >= 0)
    assert set(gc["kind"].tolist()) == set(range(9))
    c = 5
    ns = inp["nstar"][:, c]
    for r in range(nrec):
        up, dn = _by_hand(sq, atom, inp, c, r, ns[gc["ll"][r]], ns[gc["ul"][r]])
        assert cup[r0 + r, c] == pytest.approx(up, rel=1e-13, abs=0), r
        assert cup[r0 + nrec + r, c] == pytest.approx(dn, rel=1e-13, abs=0), r
    # where n*_ll = 0 the ratio comes from the Saha term
    nstar = inp["nstar"].copy()
    nstar[gc["ll"], c] = 0.0
    cup0 = _rates(sq, atom, inp, nstar)
    for r in range(nrec):
        up, dn = _by_hand(sq, atom, inp, c, r, 0.0, nstar[gc["ul"][r], c])
        assert cup0[r0 + r, c] == pytest.approx(up, rel=1e-12, abs=0), r
        assert cup0[r0 + nrec + r, c] == pytest.approx(dn, rel=1e-12, abs=0), r
    # the classic rows do not read the records
    plain = dict(atom, gencol=None)
    assert np.array_equal(cup[:r0], sq.collision_rates(plain, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"]))


def test_rate_matrix_adds_records_after_classic(sq):
    from test_stateq_oracle import _numpy_rate_matrix
    atom, inp = _case(ncell=32)
    cup = _rates(sq, atom, inp)
    gc = atom["gencol"]
    ncol, nrec = len(atom["col_i"]), len(gc["ll"])
    n = atom["nlevel"]
    for c in (0, 13, 31):
        # an independent assembly: the radiative matrix of the atom without
        # collisions plus the collision matrix c, scaled as the rate matrix is
        ns = inp["nstar"][:, c]
        w, e = sq.rate_matrix(atom, inp, c, cup)
        cm = np.zeros((n, n))
        for p in range(ncol):
            i, j = atom["col_i"][p], atom["col_j"][p]
            for u in (cup[p, c], cup[ncol + p, c]):
                if u != 0:
                    cm[j, i] += u
                    cm[i, j] += u * ns[i] / ns[j]
        for r in range(nrec):
            cm[gc["ul"][r], gc["ll"][r]] += cup[2 * ncol + r, c]
            cm[gc["ll"][r], gc["ul"][r]] += cup[2 * ncol + nrec + r, c]
        plain = dict(atom, gencol=None, col_hkind=None, col_i=np.zeros(0, np.int32), col_j=np.zeros(0, np.int32),
                     col_kind=np.zeros(0, np.int32), col_fac=np.zeros(0, np.float32))
        wr, er = _numpy_rate_matrix(plain, inp, c, np.zeros((0, inp["temp"].size)))
        bl = inp["b"][:, c]
        pos = int(np.argmax(bl * ns))
        cmd = cm - np.diag(cm.sum(axis=0))
        add = cmd * (bl * ns)[None, :]
        add[pos] = 0
        wr = wr + add
        scale = np.abs(wr).max(axis=0, keepdims=True)
        assert np.max(np.abs(w - wr) / scale) < 1e-12
        assert np.array_equal(e, er)


@pytest.mark.parametrize("solver", [0, 2])
def test_lte_gives_b_one_with_records(sq, solver):
    atom, inp = _case(ncell=256, lte=True)
    cup = _rates(sq, atom, inp)
    b = inp["b"].copy()
    res, lvlerr, rc = sq.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                       inp["gamma_ji"], temp=inp["temp"], cup=cup, solver=solver)
    assert rc == 0 and np.max(np.abs(b - 1.0)) < 2e-6

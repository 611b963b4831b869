"""Hydrogen collision recipes of classic_col in the SE oracle (CPU only).

  * prepare_Drawin's prefactor (atom_mod.f90:1741-1750): the host restatement in
    dispatch_b200.stateq and the oracle agree bit for bit, and its constant
    16 pi a0^2 is the 1.40758e-15 cm^2 the reference quotes;
  * Drawin's and Takeda's rates (atom_mod.f90:1854-1876) of one pair and cell
    worked by hand;
  * the hydrogen rows leave the electron rows as they were;
  * the pair selection of classic_col (classic_pairs) against model_atom's list;
  * the rate matrix takes c(j,i) = u_e + u_h and c(i,j) = (u_e + u_h) n*_i/n*_j;
  * hydrogen collisions keep detailed balance: LTE still gives b = 1.
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
    return synth.se_config("small", ncell=ncell, h_recipes=H_RECIPES, **kw)


def test_prepare_drawin_host_matches_oracle(sq):
    for awgt in (1.008, 4.003, 23.0, 40.08, 55.847, 137.33):
        assert stateq.prepare_drawin(awgt) == sq.prepare_drawin(awgt)
    assert 16 * math.pi * 5.29177349e-9**2 == pytest.approx(1.40758e-15, rel=1e-5)
    # the prefactor of hydrogen itself (A = 1.008), worked by hand
    mu_h = 1.0 / 2.008
    ame = float(np.float32(5.485799e-4))
    v = 16 * math.pi * 5.29177349e-9**2 * math.sqrt(2 * 1.380662e-16 / (math.pi * 1.6726e-24 * 1.008 * mu_h))
    assert stateq.prepare_drawin(1.008) == pytest.approx(v * ame / (ame + 1.0) / mu_h, rel=1e-14)


def test_kinds_follow_the_recipes():
    atom, _ = _case()
    cont = atom["ion"][atom["col_j"]] > atom["ion"][atom["col_i"]]
    no_f = atom["col_fac"] == 0
    hk = atom["col_hkind"]
    assert np.all(hk[~cont & no_f] == stateq.COLH_TAKEDA)
    assert np.all(hk[cont | ~no_f] == stateq.COLH_DRAWIN)
    assert np.any(hk == stateq.COLH_TAKEDA) and np.any(hk == stateq.COLH_DRAWIN)
    only = synth.model_atom(5, h_recipes=("drawin", "", ""))
    c2 = only["ion"][only["col_j"]] > only["ion"][only["col_i"]]
    assert np.all(only["col_hkind"][~c2] == 1) and np.all(only["col_hkind"][c2] == 0)


def test_drawin_and_takeda_by_hand(sq):
    atom, inp = _case(ncell=32)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    ncol = len(atom["col_i"])
    assert cup.shape == (2 * ncol, 32) and np.all(np.isfinite(cup)) and np.all(cup >= 0)
    ame = float(np.float32(5.485799e-4))
    mu_e = ame / (ame + 1.0)
    drawin = stateq.prepare_drawin(atom["awgt"])
    c = 7
    T, ne, ekt, nh1 = inp["temp"][c], inp["ne"][c], inp["e_kT"][c], inp["nh1"][c]
    c0 = math.pi * (5.29177349e-9 * 5.29177349e-9) * math.sqrt(8 * 1.380662e-16 / 9.109534e-28 / math.pi)
    rydk = 13.605 * (1.602189e-12 / 1.380662e-16)
    allen = c0 * rydk * ne / math.sqrt(T)
    hk = atom["col_hkind"]
    for kind in (stateq.COLH_DRAWIN, stateq.COLH_TAKEDA):
        for p in np.flatnonzero(hk == kind)[:4]:
            i, j = atom["col_i"][p], atom["col_j"][p]
            cont = atom["ion"][j] > atom["ion"][i]
            dev = max(atom["ev"][j] - atom["ev"][i], 1e-8)
            u0 = dev * ekt
            ex = math.exp(-u0)
            if kind == stateq.COLH_TAKEDA:
                v = nh1 * (allen / ne) * int(atom["ion"][i]) / atom["g"][i] * ex * math.sqrt(ame)
            else:
                t = 2.0 / u0
                t = (1.0 + t) / (1.0 + (mu_e * t) ** 2)
                v = nh1 * drawin * (13.605 / dev) ** 2 * t * ex * math.sqrt(T)
                if not cont:
                    v *= max(float(atom["col_fac"][p]), float(np.float32(1e-6)) * atom["g"][j])
            assert cup[ncol + p, c] == pytest.approx(v, rel=1e-13), (kind, p)
    # the electron rows are those of the atom without hydrogen recipes
    plain = dict(atom, col_hkind=None)
    ref = sq.collision_rates(plain, inp["temp"], inp["ne"], inp["e_kT"])
    assert np.array_equal(cup[:ncol], ref)
    # nh1 scales the hydrogen rows and nothing else
    cup2 = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=2 * inp["nh1"])
    assert np.array_equal(cup2[:ncol], cup[:ncol])
    np.testing.assert_allclose(cup2[ncol:], 2 * cup[ncol:], rtol=1e-15)


def test_hydrogen_only_pairs_and_colscale(sq):
    atom, inp = _case(ncell=16)
    ncol = len(atom["col_i"])
    a2 = dict(atom, col_kind=np.zeros(ncol, np.int32), colscale=3.0, cbbhsc=0.5, cbfhsc=2.0)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    cup2 = sq.collision_rates(a2, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    assert np.all(cup2[:ncol] == 0)
    cont = atom["ion"][atom["col_j"]] > atom["ion"][atom["col_i"]]
    fac = np.where(cont, 2.0, 0.5)[:, None] * 3.0
    np.testing.assert_allclose(cup2[ncol:], cup[ncol:] * fac, rtol=1e-15)


def test_classic_pairs_reproduce_model_atom():
    for rec in (None, H_RECIPES, ("", "drawin", "")):
        atom = synth.model_atom(3, nbound=12, nline=20, h_recipes=rec)
        n = atom["nlevel"]
        cdata = np.zeros((n, n), np.float32)
        cdata[atom["col_i"], atom["col_j"]] = atom["col_fac"]
        cont_up = np.where(atom["ion"] == 1, n - 1, -1)
        h = rec or ("", "", "")
        got = stateq.classic_pairs(atom["ion"], cont_up, cdata, h_excitation=h[0], h_ionisation=h[1],
                                   h_forbidden=h[2])
        for k in ("col_i", "col_j", "col_kind", "col_fac"):
            assert np.array_equal(got[k], atom[k]), k
        if atom["col_hkind"] is None:
            assert got["col_hkind"] is None
        else:
            assert np.array_equal(got["col_hkind"], atom["col_hkind"])
    # data in the file removes a recipe; a pair with both kinds of data is left out
    ecol = np.zeros((n, n), bool)
    hcol = np.zeros((n, n), bool)
    ecol[0, 1] = hcol[0, 1] = True
    ecol[0, 2] = True
    got = stateq.classic_pairs(atom["ion"], cont_up, cdata, ecol=ecol, hcol=hcol, h_excitation="drawin")
    pairs = list(zip(got["col_i"], got["col_j"]))
    assert (0, 1) not in pairs
    p = pairs.index((0, 2))
    assert got["col_kind"][p] == 0 and got["col_hkind"][p] == stateq.COLH_DRAWIN


def test_rate_matrix_sums_electron_and_hydrogen(sq):
    from test_stateq_oracle import _numpy_rate_matrix
    atom, inp = _case(ncell=64)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    ncol = len(atom["col_i"])
    for c in (0, 17, 63):
        w, e = sq.rate_matrix(atom, inp, c, cup)
        wr, er = _numpy_rate_matrix(atom, inp, c, cup[:ncol] + cup[ncol:])
        scale = np.abs(wr).max(axis=0, keepdims=True)
        assert np.max(np.abs(w - wr) / scale) < 1e-13
        assert np.array_equal(e, er)
        # the hydrogen rates change the matrix
        w0, _ = sq.rate_matrix(dict(atom, col_hkind=None), inp, c, cup[:ncol])
        assert not np.array_equal(w, w0)


@pytest.mark.parametrize("solver", [0, 2])
def test_lte_gives_b_one_with_hydrogen(sq, solver):
    atom, inp = _case(ncell=256, lte=True)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"], nh1=inp["nh1"])
    b = inp["b"].copy()
    res, lvlerr, rc = sq.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                       inp["gamma_ji"], temp=inp["temp"], cup=cup, solver=solver)
    assert rc == 0 and np.max(np.abs(b - 1.0)) < 2e-6

"""The statistical-equilibrium oracle against known answers (CPU only).

  * expin against scipy's E1: the reference's rational approximations with
    single-precision coefficients (atom_mod.f90:2362-2397) stay within 5e-6;
  * the three dense solvers against numpy's LAPACK solve; lineq's full
    pivoting on a matrix with a zero pivot (op_math_mod.f90:263-356);
  * the rate matrix of a cell against an independent numpy assembly of
    setup_transition_matrix (atom_mod.f90:740-841);
  * LTE: a Planck radiation field puts every transition in detailed balance,
    so b = 1 solves the rate equations whatever b the update starts from;
  * particle conservation sum(b n*) = totn, and the rate equations satisfied by
    the new populations (update_populations :439-732);
  * Ng: ln b iterates with exactly two geometric modes extrapolate exactly to
    the limit (ng_mod.f90:1-23);
  * the Ng gate's conditions in order (ng_mod.f90:153-215).
"""
import math

import numpy as np
import pytest

from dispatch_b200 import synth
from dispatch_b200.stateq import NgParams, NgState


@pytest.fixture(scope="module")
def sq(oracle):
    from oracle import stateq
    return stateq


def test_expin_matches_e1(sq):
    special = pytest.importorskip("scipy.special")
    x = np.concatenate([np.logspace(-6, 0, 200), np.linspace(1.0, 4.0, 200)[1:], np.linspace(4.0, 80.0, 300)[1:]])
    got = sq.expin(x)
    ref = special.exp1(x)
    assert np.max(np.abs(got / ref - 1.0)) < 5e-6
    assert sq.expin(np.array([0.0, -1.0])).tolist() == [0.0, 0.0]


@pytest.mark.parametrize("solver", [0, 1, 2])
def test_dense_solvers(sq, solver):
    rng = np.random.default_rng(11)
    for n in (1, 2, 5, 21, 61):
        a = rng.standard_normal((n, n)) + n * np.eye(n)
        b = rng.standard_normal(n)
        x = sq.solve(a, b, solver)
        assert np.allclose(x, np.linalg.solve(a, b), rtol=1e-11, atol=1e-13)


def test_full_pivot_zero_diagonal(sq):
    a = np.array([[0.0, 2.0, 1.0], [1.0, 0.0, 3.0], [4.0, 1.0, 0.0]])
    b = np.array([1.0, 2.0, 3.0])
    ref = np.linalg.solve(a, b)
    assert np.allclose(sq.solve(a, b, 1), ref, rtol=1e-14)
    assert np.allclose(sq.solve(a, b, 2), ref, rtol=1e-14)
    assert not np.all(np.isfinite(sq.solve(a, b, 0)))


def _numpy_rate_matrix(atom, inp, c, cup, cut_x=70.0):
    n = atom["nlevel"]
    bl, ns = inp["b"][:, c], inp["nstar"][:, c]
    w = np.zeros((n, n))
    for kr in range(len(atom["ti"])):
        i, j = atom["ti"][kr], atom["tj"][kr]
        if (atom["ev"][j] - atom["ev"][i]) * inp["e_kT"][c] > cut_x:
            cr = atom["Aji"][kr] if kr < atom["nline"] else 1.0
            w[i, j] += cr
            w[j, i] += cr * ns[j] / ns[i]
            continue
        th, dv = float(inp["gamma_ij"][kr, c]), float(inp["gamma_ji"][kr, c])
        if kr < atom["nline"]:
            gij = atom["g"][i] / atom["g"][j]
            beta = ns[j] * gij / ns[i]
            up, dn = th * beta / (1 - beta) + dv, gij * (th / (1 - beta) + dv)
        else:
            up, dn = th, dv
        w[j, i] += up
        w[i, j] += dn
    for p in range(len(atom["col_i"])):
        i, j = atom["col_i"][p], atom["col_j"][p]
        w[j, i] += cup[p, c]
        w[i, j] += cup[p, c] * ns[i] / ns[j]
    w -= np.diag(w.sum(axis=0))
    pos = int(np.argmax(bl * ns))
    w = w * (bl * ns)[None, :]
    w[pos] = bl * ns
    e = np.zeros(n)
    e[pos] = inp["totn"][c]
    return w, e


def test_rate_matrix_matches_numpy(sq):
    atom, inp = synth.se_config("small", ncell=64)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    for c in (0, 17, 63):
        w, e = sq.rate_matrix(atom, inp, c, cup)
        wr, er = _numpy_rate_matrix(atom, inp, c, cup)
        scale = np.abs(wr).max(axis=0, keepdims=True)
        assert np.max(np.abs(w - wr) / scale) < 1e-13
        assert np.array_equal(e, er)


def test_collisions_regemorter_seaton(sq):
    special = pytest.importorskip("scipy.special")
    atom, inp = synth.se_config("small", ncell=32)
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    assert np.all(cup >= 0) and np.all(np.isfinite(cup))
    # van Regemorter by hand for one bound pair and one cell
    p = int(np.flatnonzero(atom["col_kind"] == 1)[3])
    i, j, c = atom["col_i"][p], atom["col_j"][p], 5
    T, ne, ekt = inp["temp"][c], inp["ne"][c], inp["e_kT"][c]
    dev = max(atom["ev"][j] - atom["ev"][i], 1e-8)
    f = max(float(atom["col_fac"][p]), float(np.float32(1e-6)) * atom["g"][j])
    u0 = dev * ekt
    c0 = math.pi * 5.29177349e-9**2 * math.sqrt(8 * 1.380662e-16 / 9.109534e-28 / math.pi)
    rydk = 13.605 * 1.602189e-12 / 1.380662e-16
    allen = c0 * rydk * ne / math.sqrt(T)
    v = 14.5 * allen * rydk / (1.602189e-12 / 1.380662e-16) * f * max(0.2 * math.exp(-u0),
                                                                        math.sqrt(3) / 2 / math.pi * special.exp1(u0)) / dev
    assert cup[p, c] == pytest.approx(v, rel=1e-5)


def _update(sq, atom, inp, solver=0, **kw):
    cup = sq.collision_rates(atom, inp["temp"], inp["ne"], inp["e_kT"])
    b = inp["b"].copy()
    res, lvlerr, rc = sq.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                       inp["gamma_ji"], temp=inp["temp"], cup=cup, solver=solver, **kw)
    return b, res, lvlerr, rc, cup


@pytest.mark.parametrize("solver", [0, 1, 2])
def test_lte_gives_b_one(sq, solver):
    atom, inp = synth.se_config("small", ncell=256, lte=True)
    b, res, lvlerr, rc, _ = _update(sq, atom, inp, solver)
    assert rc == 0 and res["nclamp"] == 0 and res["ntot"] == 256 * atom["nlevel"]
    assert np.max(np.abs(b - 1.0)) < 2e-6
    # the largest change is the start perturbation undone
    assert res["maxerr"] == lvlerr[res["epos_level"]] or abs(res["maxerr"]) <= np.max(np.abs(lvlerr))


def test_conservation_and_rate_equations(sq):
    atom, inp = synth.se_config("small", ncell=256)
    b, res, lvlerr, rc, cup = _update(sq, atom, inp)
    assert rc == 0
    assert np.allclose((b * inp["nstar"]).sum(axis=0), inp["totn"], rtol=1e-13)
    # the new populations solve the unscaled rate equations in every row but the conservation one
    for c in (0, 100, 255):
        # with b = 1 the helper returns R(i, j) n*_j, its conservation row at argmax n*
        w, _ = _numpy_rate_matrix(atom, dict(inp, b=np.ones_like(inp["b"])), c, cup)
        r = w @ b[:, c]
        mag = np.abs(w) @ np.abs(b[:, c])
        r[int(np.argmax(inp["nstar"][:, c]))] = 0
        r[int(np.argmax(inp["b"][:, c] * inp["nstar"][:, c]))] = 0
        assert np.max(np.abs(r) / mag) < 1e-9


def test_solvers_agree(sq):
    atom, inp = synth.se_config("small", ncell=128)
    b0 = _update(sq, atom, inp, 0)[0]
    for s in (1, 2):
        bs = _update(sq, atom, inp, s)[0]
        assert np.max(np.abs(bs / b0 - 1)) < 1e-9


def test_limiter_and_skips(sq):
    atom, inp = synth.se_config("small", ncell=64)
    inp = dict(inp)
    b = inp["b"].copy()
    b[3, :8] *= 1e-6          # far from the solution: the correction is clamped
    inp["b"] = b
    totn = inp["totn"].copy()
    totn[10] = 0.0            # no atoms: left alone
    inp["totn"] = totn
    temp = inp["temp"].copy()
    temp[11] = 2e7            # above tmax_update: left alone
    inp["temp"] = temp
    bn, res, _, rc, _ = _update(sq, atom, inp)
    assert rc == 0 and res["nclamp"] >= 8 and res["ntot"] == 62 * atom["nlevel"]
    assert np.array_equal(bn[:, 10], b[:, 10]) and np.array_equal(bn[:, 11], b[:, 11])
    # the limited correction saturates towards 2 max_update (times the renormalisation)
    ratio = bn[3, :8] / b[3, :8]
    assert np.all((ratio > 150) & (ratio < 2 * 100 * 1.05))


def test_nonfinite_cell_left_alone(sq):
    atom, inp = synth.se_config("small", ncell=16)
    inp = dict(inp)
    g = inp["gamma_ij"].copy()
    g[0, 5] = np.nan
    inp["gamma_ij"] = g
    bn, res, _, rc, _ = _update(sq, atom, inp)
    assert rc == 5 and res["nonfinite_cell"] == 5
    assert np.array_equal(bn[:, 5], inp["b"][:, 5])


def test_ng_two_modes_exact(sq):
    rng = np.random.default_rng(3)
    nlevel, ncell = 6, 50
    xinf = rng.normal(0, 0.5, (nlevel, ncell))
    v1, v2 = rng.normal(0, 0.1, (2, nlevel, ncell))
    r1, r2 = 0.8, 0.5
    it = [np.exp(xinf + r1**k * v1 + r2**k * v2) for k in range(4)]
    oldb = np.ascontiguousarray(np.stack(it[:3]))
    b = np.ascontiguousarray(it[3])
    gram = sq.ng_accumulate(b, oldb)
    st = NgState()
    st.d_done = gram[:6].copy()
    st.coefficients()
    nstar = np.ones((nlevel, ncell))
    totn = np.exp(xinf).sum(axis=0)
    out = sq.ng_extrapolate(b, oldb, nstar, totn, st.a, st.b)
    assert out["applied"]
    assert np.max(np.abs(np.log(b) - xinf)) < 1e-9
    # veto: a step larger than max_change leaves b alone
    b2 = np.ascontiguousarray(it[3])
    out = sq.ng_extrapolate(b2, oldb, nstar, totn, st.a, st.b, max_change=1e-6)
    assert not out["applied"] and np.array_equal(b2, it[3])


def test_ng_gate_order():
    st = NgState(params=NgParams())
    assert st.should_fire(5, 1.0, 1e-3) == (False, "no-history")
    st.s_done, st.s_prev = 1.0, 2.0
    st.iter_fired = 3
    assert st.should_fire(5, 1.0, 1e-3) == (False, "min-gap")
    st.iter_fired = -10**9
    st.ntot_done, st.nclamp_done = 1000, 5
    assert st.should_fire(5, 1.0, 1e-3) == (False, "clamped")
    st.nclamp_done = 0
    st.r, st.r_prev = 0.8, -1.0
    assert st.should_fire(5, 1.0, 1e-3) == (False, "not-stationary")
    st.r_prev = 0.5
    assert st.should_fire(5, 1.0, 1e-3) == (False, "not-stationary")
    st.r, st.r_prev = 0.3, 0.31
    assert st.should_fire(5, 1.0, 1e-3) == (False, "fast-enough")
    st.r, st.r_prev = 1.1, 1.05
    assert st.should_fire(5, 1.0, 1e-3) == (False, "diverging")
    st.r, st.r_prev = 0.8, 0.82
    assert st.should_fire(5, 1e-3, 1e-3) == (False, "no-headroom")
    st.d_done = np.array([0.0, 0.0, 1.0, 1.0, 1.0, 1.0])   # d1 parallel to d2
    assert st.should_fire(5, 1.0, 1e-3) == (False, "ill-conditioned")
    st.d_done = np.array([0.3, 0.1, 1.0, 0.2, 0.2, 1.0])
    assert st.should_fire(5, 1.0, 1e-3) == (True, "FIRE")


def test_ng_promote_rate():
    st = NgState()
    st.add_gram(np.array([0, 0, 0, 0, 0, 0, 4.0]))
    st.promote(3)
    assert st.r == -1.0 and st.s_prev == 4.0
    st.add_gram(np.array([0, 0, 0, 0, 0, 0, 1.0]))
    st.promote(4)
    assert st.r == pytest.approx(0.5) and st.r_prev == -1.0
    st.promote(4)          # idempotent within an iteration
    assert st.r == pytest.approx(0.5)
    st.promote(5)          # an empty accumulation leaves the rate stale
    assert st.r == pytest.approx(0.5) and st.s_prev == 1.0

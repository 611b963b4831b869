"""The model-atom opacity and rate oracle against known answers (CPU only).

  * the split tracking holds every contribution: largest + rest equals the
    running total up to the order of the float additions, and the tracked
    index is the contribution of largest magnitude (add_largest,
    rt_patch_mod.f90:3150-3187);
  * a Planck field I = J = B_nu puts each line's and continuum's radiative
    rates in detailed balance: the deviation integral of the 'largest'
    formulation is exactly zero, that of the 'original' one zero to float
    rounding, and a continuum's two sums agree (bound_bound_rates
    :2869-2888, bound_free_rates :3193-3259);
  * normalize_profiles inverts wphi once and scales the rates
    (atom_mod.f90:377-430).
"""
import numpy as np
import pytest

from tests import nlte_cases


@pytest.fixture(scope="module")
def nl(oracle):
    from oracle import nlte
    return nlte


@pytest.fixture(scope="module")
def base():
    return nlte_cases.case(ncell=64)


def _opacity(nl, win, c, field, split=True):
    n, nf = c["pop_ratio"].size, win["nf"]
    adamp = nl.bb_damping(win, c["ne"], c["tothi"], c["vbar2"], c["stark_pe"], c["unsold"], c["inv_df"])
    xh, eh = field["xhat"].copy(), field["ehat"].copy()
    nl.bf_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], xh, eh)
    sp = None
    if split:
        z = lambda dt: np.zeros((n, nf), dt)
        sp = {"opac_L": z(np.float32), "opac_R": z(np.float32), "id": z(np.int32),
              "chi_L": z(np.float32), "chi_R": z(np.float32), "chi_id": z(np.int32)}
    x0, e0 = xh.copy(), eh.copy()
    nl.bb_opacity(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, xh, eh,
                  split=sp)
    return adamp, x0, e0, xh, eh, sp


def test_split_tracking_holds_the_total(nl, base):
    atom, inp, win, c, field = base
    adamp, x0, e0, xh, eh, sp = _opacity(nl, win, c, field)
    tot_e = sp["opac_L"].astype(np.float64) + sp["opac_R"]
    tot_x = sp["chi_L"].astype(np.float64) + sp["chi_R"]
    assert np.max(np.abs(tot_e / eh - 1)) < 1e-5
    assert np.max(np.abs(tot_x / xh - 1)) < 1e-5
    # points without a line keep the background as the largest (index 0)
    covered = np.zeros(win["nf"], bool)
    for b_, r_ in zip(win["line_blue"], win["line_red"]):
        covered[b_:r_ + 1] = True
    assert np.all(sp["id"][:, ~covered] == 0) and np.all(sp["opac_R"][:, ~covered] == 0)
    assert np.any(sp["id"][:, covered] > 0)


def _inv_nref(win, c):
    li, lj = win["line_i"], win["line_j"]
    beta_ref = c["nstar"][lj] * win["g"][li][:, None] / (c["nstar"][li] * win["g"][lj][:, None])
    return (1 - beta_ref) / beta_ref


def test_planck_field_detailed_balance(nl, base):
    atom, inp, win, c, field = base
    adamp, x0, e0, xh, eh, sp = _opacity(nl, win, c, field)
    n, ntr, L = c["pop_ratio"].size, win["nline"] + win["ncont"], win["nline"]
    inu = field["Bnu"]
    # 'largest' without preconditioning: dev = sum vvv (I - Bnu) = 0 exactly
    gij, gji = np.zeros((ntr, n), np.float32), np.zeros((ntr, n), np.float32)
    nl.bb_rates(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, inu,
                field["beta"], field["Bnu"], gij, gji, split_rates=True, preconditioning=False)
    assert np.all(gij[:L] > 0) and np.all(gji[:L] == 0)
    # 'original' without preconditioning: dev = sum_I - th/inv_nref, zero to float rounding of sum_I
    gij2, gji2 = np.zeros_like(gij), np.zeros_like(gji)
    nl.bb_rates(win, c["b"], c["nstar"], c["pop_ratio"], c["e_kT"], c["inv_df"], c["vproj"], adamp, inu,
                field["beta"], field["Bnu"], gij2, gji2, psi=field["psi"], split_rates=False, preconditioning=False)
    sum_i = gij2[:L] / _inv_nref(win, c)
    assert np.max(np.abs(gji2[:L]) / sum_i) < 1e-5
    # the two formulations' thermal parts agree
    assert np.max(np.abs(gij2[:L].astype(np.float64) / gij[:L] - 1)) < 1e-5
    # continua: with J = Bnu = beta/(1 - beta), beta (J + 1) = J and the two sums agree
    gbi, gbj = np.zeros_like(gij), np.zeros_like(gji)
    nl.bf_rates(win, c["b"], c["nstar"], c["e_kT"], inu, field["psi"], field["beta"], gbi, gbj,
                preconditioning=False)
    k = slice(L, ntr)
    assert np.all(gbi[k] > 0)
    assert np.max(np.abs(gbj[k].astype(np.float64) / gbi[k] - 1)) < 1e-4


def test_normalize_profiles(nl):
    rng = np.random.default_rng(1)
    atom = {"ti": np.array([0, 1, 0, 1], np.int32), "tj": np.array([1, 2, 3, 3], np.int32), "nline": 2,
            "active": None}
    n = 16
    nstar = np.exp(rng.normal(0, 1, (4, n)))
    wphi = rng.random((2, n)).astype(np.float32)
    wphi[0, 3] = 0.0
    gij = rng.random((4, n)).astype(np.float32)
    gji = rng.random((4, n)).astype(np.float32)
    g0, j0, w0 = gij.copy(), gji.copy(), wphi.copy()
    nl.normalize_profiles(atom, nstar, wphi, gij, gji, np.array([1, 0], np.uint8), True)
    with np.errstate(divide="ignore"):
        inv = np.where(w0[0] > 0, np.float32(1) / w0[0], np.float32(1))
    assert np.array_equal(wphi[0], inv) and np.array_equal(wphi[1], w0[1])
    assert np.array_equal(gij[0], g0[0] * inv) and np.array_equal(gij[1], g0[1])
    ratio = nstar[[0, 1]] / nstar[[3, 3]]
    assert np.array_equal(gji[2:], (j0[2:].astype(np.float64) * ratio).astype(np.float32))

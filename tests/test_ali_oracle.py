"""Host-side checks of the ALI pieces that need no GPU: the quadratures of the
iteration (mean-intensity weights, Gauss-Radau), the transition subsets of a
frequency window, and the oracle's composition of the iteration itself."""
import math

import numpy as np
import pytest


def test_radau_rule_known_answers():
    from dispatch_b200 import synth
    mu, w = synth.radau_nodes(2)
    # x = -1, 1/3 on [-1, 1] with weights 1/2, 3/2 (radau_mod.f90 row 2)
    np.testing.assert_array_equal(mu, np.float32([1.0 - (0.5 + 0.5 / 3.0), 1.0]))
    np.testing.assert_array_equal(w, np.float32([0.75, 0.25]))
    for k in range(1, 11):
        mu, w = synth.radau_nodes(k)
        assert mu[-1] == 1.0 and np.all(np.diff(mu) > 0)
        # exact for polynomials of degree 2k - 2 on [0, 1]
        for p in range(2 * k - 1):
            assert float(np.sum(w.astype(np.float64) * mu.astype(np.float64) ** p)) == pytest.approx(
                1.0 / (p + 1), rel=2e-6, abs=2e-7)
    with pytest.raises(ValueError):
        synth.radau_nodes(11)


@pytest.mark.parametrize("kind", ["lobatto", "gauss", "radau"])
def test_mean_intensity_weights(kind):
    from dispatch_b200 import synth
    fn = {"lobatto": lambda j: synth.lobatto_rays(4, 4, jnu_weights=j),
          "gauss": lambda j: synth.gauss_rays(3, 4, jnu_weights=j),
          "radau": lambda j: synth.radau_rays(3, 4, jnu_weights=j)}[kind]
    vec, w = fn(True)
    n = vec.shape[0] // 2
    np.testing.assert_array_equal(vec[n:], -vec[:n])
    np.testing.assert_array_equal(w[n:], w[:n])
    assert w.sum() == pytest.approx(1.0, abs=1e-6)
    assert np.all(vec[:n, 2] > 0)
    np.testing.assert_allclose(np.linalg.norm(vec, axis=1), 1.0, atol=2e-3)
    fv, fw = fn(False)
    np.testing.assert_array_equal(fv, vec[:n])
    np.testing.assert_allclose(fw, 2.0 * w[:n] * vec[:n, 2])


def test_radau_azimuths_rotated():
    from dispatch_b200 import synth
    vec, _ = synth.radau_rays(2, 4)
    # mu = 1 once, then four azimuths from pi/4 (zrot)
    assert vec.shape == (5, 3)
    np.testing.assert_array_equal(vec[0], [0.0, 0.0, 1.0])
    phi = np.arctan2(vec[1:, 1], vec[1:, 0]) % (2 * math.pi)
    np.testing.assert_allclose(phi, np.array([1, 3, 5, 7]) * math.pi / 4, atol=1e-9)


def test_window_subsets_partition_the_atom():
    from dispatch_b200 import synth
    atom = synth.model_atom(2, nbound=6, nline=8)
    full = synth.atom_window(atom)
    nrad = len(atom["ti"])
    parts = [list(range(0, nrad, 2)), list(range(1, nrad, 2))]
    got_l, got_c = [], []
    for p in parts:
        w = synth.atom_window(atom, transitions=p)
        got_l += list(w["line_ntrans"])
        got_c += list(w["cont_ntrans"])
        assert w["line_red"].max(initial=0) < w["nf"] and w["cont_red"].max(initial=0) < w["nf"]
        # a line keeps its damping and its Einstein coefficients
        np.testing.assert_array_equal(w["grad"], full["grad"][w["line_ntrans"]])
        np.testing.assert_array_equal(w["Aij"], full["Aij"][w["line_ntrans"]])
        np.testing.assert_array_equal(w["line_index"], w["line_ntrans"] + 1)
    assert sorted(got_l) == list(range(atom["nline"]))
    assert sorted(got_c) == list(range(atom["nline"], nrad))


@pytest.fixture(scope="module")
def oracle_run():
    from dispatch_b200 import ali
    from oracle import ali as oali
    from oracle import oracle as O
    O.build()
    cube, atom, win, vec, wts = ali.cube_problem(nx=4, ny=4, nz=8, nbound=4, nline=4, ntheta=2, nphi=2)
    hist, S = oali.run(cube, atom, win, vec, wts, maxiter=6, convlim=1e-6)
    return hist, S


def test_oracle_ali_conserves_and_contracts(oracle_run):
    hist, S = oracle_run
    assert len(hist) == 6
    np.testing.assert_allclose((S["b"] * S["nstar"]).sum(axis=0), S["totn"], rtol=1e-12)
    err = [abs(h["maxerr"]) for h in hist]
    assert err[-1] < err[0]
    assert np.all(np.isfinite(S["J"])) and np.all(S["J"] >= 0)
    # the twins are combined: both hemispheres hold the mean intensity
    np.testing.assert_array_equal(S["J"][0], S["J"][1])


def test_column_set_layout():
    from dispatch_b200 import synth
    c = synth.column_set(3, ncol=5, depth=(6, 9), nz=12, nxy=3, variants=(0.0, 0.2))
    off = c["col_off"]
    assert off[0] == 0 and off[-1] == c["temp"].size and len(off) == 11
    d = np.diff(off)
    assert d.min() >= 6 and d.max() <= 9
    # the second variant repeats the columns with the abundance offset
    np.testing.assert_array_equal(d[:5], d[5:])
    np.testing.assert_array_equal(c["temp"][:off[5]], c["temp"][off[5]:])
    assert np.all(c["abund_dex"][off[5]:] == 0.2) and np.all(c["abund_dex"][:off[5]] == 0.0)
    # each column runs bottom to top: the temperature falls upwards on average
    assert np.mean([c["temp"][off[k]] > c["temp"][off[k + 1] - 1] for k in range(10)]) > 0.5


def test_oracle_columns_conserve_and_contract():
    from dispatch_b200 import ali
    from oracle import ali as oali
    from oracle import oracle as O
    O.build()
    cols, atom, wins, mu, wmu = ali.column_problem(ncol=4, depth=(6, 10), nz=12, nxy=3, nbound=4, nline=4)
    hist, S = oali.run_columns(cols, atom, wins, mu, wmu, maxiter=5, convlim=1e-6)
    np.testing.assert_allclose((S["b"] * S["nstar"]).sum(axis=0), S["totn"], rtol=1e-12)
    err = [abs(h["maxerr"]) for h in hist]
    assert err[-1] < err[0]
    np.testing.assert_array_equal(S["J"][0], S["J"][1])

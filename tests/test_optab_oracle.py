"""The sampled opacity table oracle (oracle/or_optab.c) against the contracts of
HOP/optab_mod.f90 and interpol_mod.f90 and the interpolation requirements the
reference tests for its grid interpolation (tests/science/test_interpolation.py):
node slopes equal to an independent numpy restatement bit for bit; a query on a
node returns the node; constant and linear fields are reproduced off the nodes; a
monotone field stays inside its bracketing nodes on interior intervals; the
scattering part never exceeds the total; the line-list query is the unshifted one
at lam (1 + vproj).  No golden vectors of the reference exist for this path, so
these properties are its pins."""
import numpy as np
import pytest

import optab_cases as oc


def test_slopes_match_numpy_restatement(oracle):
    from oracle import optab
    for kind in ("background", "linelist"):
        tab = oc.table(kind, nnu=120)
        for comp in ("val", "scat"):
            dl, dt, de = optab.slopes(tab, comp)
            p = tab["pca"]
            np.testing.assert_array_equal(dl, oc.slopes_lam(tab["lam"], tab[comp]))
            np.testing.assert_array_equal(dt, oc.slopes_axis(p["c0"][0], p["dc"][0], tab[comp], 1))
            np.testing.assert_array_equal(de, oc.slopes_axis(p["c0"][1], p["dc"][1], tab[comp], 0))


def test_two_node_axes(oracle):
    """Two nodes on an axis: both slopes are the secant (pchip_slopes, n == 2)."""
    from oracle import optab
    tab = oc.table("background", nnu=2)
    dl, _, _ = optab.slopes(tab)
    sec = (tab["val"][..., 1].astype(np.float64) - tab["val"][..., 0]) / (tab["lam"][1] - tab["lam"][0])
    np.testing.assert_allclose(dl[..., 0], sec, rtol=1e-6)
    np.testing.assert_allclose(dl[..., 1], sec, rtol=1e-6)


def _with_field(tab, field):
    t = dict(tab)
    nne, ntemp, nnu = tab["val"].shape
    je, it, k = np.meshgrid(np.arange(nne), np.arange(ntemp), np.arange(nnu), indexing="ij")
    t["val"] = field(k, it, je).astype(np.float32)
    t["scat"] = (0.5 * t["val"]).astype(np.float32)
    return t


def _pc_coords(tab, T, ne):
    p = tab["pca"]
    d = np.stack([np.log(T) - p["mu"][0], np.log(ne) - p["mu"][1]])
    q = np.asarray(p["rot"]).T @ d
    return (q[0] - p["c0"][0]) / p["dc"][0], (q[1] - p["c0"][1]) / p["dc"][1]


def test_node_query_returns_the_node(oracle):
    from oracle import optab
    tab = oc.table("linelist", nnu=200)
    picks = [(3, 2), (10, 7), (40, 12)]
    T, ne = oc.node_cells(tab, picks)
    ks = np.array([5, 77, 150])
    back, scat = optab.sample(tab, T, ne, np.ones(len(picks), np.float32), tab["lam"][ks])
    for c, (it, je) in enumerate(picks):
        want = tab["val"][je, it, ks] + tab["scat"][je, it, ks]
        np.testing.assert_allclose(back[c], want, rtol=2e-5)
        np.testing.assert_allclose(scat[c], tab["scat"][je, it, ks], rtol=2e-5)


def test_constant_and_linear_fields(oracle):
    """A constant stays constant; a field linear in (lambda, PC1, PC2) is returned
    to fp32 rounding anywhere inside the grid (collinear data give every node
    the secant slope, so each cubic is the line)."""
    from oracle import optab
    c = oc.cells()
    tab = oc.table("background", nnu=150, cells_=c)
    lam = tab["lam"]
    const = _with_field(tab, lambda k, it, je: np.full(k.shape, 3.0))
    q = np.linspace(lam[3], lam[-4], 37)
    back, scat = optab.sample(const, c["temp"], c["ne"], np.ones_like(c["chi500"]), q)
    np.testing.assert_allclose(back, 4.5, rtol=1e-6)
    p = tab["pca"]
    lin = _with_field(tab, lambda k, it, je: 2.0 + 1e-3 * lam[k] + 0.1 * it + 0.2 * je)
    back, scat = optab.sample(lin, c["temp"], c["ne"], np.ones_like(c["chi500"]), q)
    u, v = _pc_coords(tab, c["temp"], c["ne"])
    want = 2.0 + 1e-3 * q[None, :] + 0.1 * u[:, None] + 0.2 * v[:, None]
    np.testing.assert_allclose(back, 1.5 * want, rtol=2e-6)


def test_monotone_field_stays_in_its_bracket(oracle):
    """tanh along each axis, queried inside interior intervals."""
    from oracle import optab
    c = oc.cells()
    tab = oc.table("background", nnu=60, cells_=c)
    nne, ntemp, nnu = tab["val"].shape
    u, v = _pc_coords(tab, c["temp"], c["ne"])
    keep = (u > 1) & (u < ntemp - 2) & (v > 1) & (v < nne - 2)
    for field, axis in ((lambda k, it, je: np.tanh((k - nnu / 2) / 4.0), "lam"),
                        (lambda k, it, je: np.tanh((it - ntemp / 2) / 3.0), "t"),
                        (lambda k, it, je: np.tanh((je - nne / 2) / 2.0), "e")):
        t = _with_field(tab, field)
        q = np.linspace(tab["lam"][2], tab["lam"][-3], 41)
        _, scat = optab.sample(t, c["temp"][keep], c["ne"][keep], np.ones(keep.sum(), np.float32), q)
        kap = scat / 0.5
        if axis == "lam":
            k = np.searchsorted(tab["lam"], q) - 1
            lo, hi = np.tanh((k - nnu / 2) / 4.0), np.tanh((k + 1 - nnu / 2) / 4.0)
            assert (kap >= lo[None, :] - 1e-6).all() and (kap <= hi[None, :] + 1e-6).all()
        else:
            x, n, s = (u[keep], ntemp, 3.0) if axis == "t" else (v[keep], nne, 2.0)
            i = np.floor(x)
            lo, hi = np.tanh((i - n / 2) / s), np.tanh((i + 1 - n / 2) / s)
            assert (kap >= lo[:, None] - 1e-6).all() and (kap <= hi[:, None] + 1e-6).all()


def test_scattering_bound_and_doppler_query(oracle):
    from oracle import optab
    c = oc.cells()
    tab = oc.table("linelist", nnu=400, cells_=c)
    q = np.linspace(4200.0, 8800.0, 96)
    back, scat = optab.sample(tab, c["temp"], c["ne"], c["chi500"], q)
    assert (scat <= back).all() and (scat >= 0).all()
    n = c["temp"].size
    v = np.full(n, 3e-5, np.float32)
    xa, ea, sa = (np.zeros((n, q.size), np.float32) for _ in range(3))
    optab.sample_ll(tab, c["temp"], c["ne"], c["chi500"], v, q, xa, ea, sa)
    xb, eb, sb = (np.zeros((n, q.size), np.float32) for _ in range(3))
    optab.sample_ll(tab, c["temp"], c["ne"], c["chi500"], np.zeros(n, np.float32), q * (1.0 + np.float64(v[0])),
                    xb, eb, sb)
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(ea, xa)
    np.testing.assert_array_equal(sa, sb)
    # the additions accumulate onto what the work slots held
    x2 = np.full((n, q.size), 1.0, np.float32)
    e2 = x2.copy()
    optab.sample_ll(tab, c["temp"], c["ne"], c["chi500"], v, q, x2, e2, None)
    np.testing.assert_array_equal(x2, np.float32(1.0) + xa)
    # and at v = 0 the line-list kappa is the value component: back - scat
    x0, e0 = (np.zeros((n, q.size), np.float32) for _ in range(2))
    optab.sample_ll(tab, c["temp"], c["ne"], c["chi500"], np.zeros(n, np.float32), q, x0, e0)
    np.testing.assert_allclose(x0, back - scat, rtol=1e-5, atol=1e-6 * back.max())

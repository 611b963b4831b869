"""The sampled opacity tables on the device (dispatch_b200.optab.SampleOptab over
m3d_optab_*) against the oracle (oracle/or_optab.c), bit for bit: the node slopes
of both components, sample_interpolate, and sample_interpolate_ll with per-cell
Doppler shifts that move queries across wavelength nodes, with and without the
scattering component, from host buffers and from device tensors."""
import numpy as np
import pytest

import optab_cases as oc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["background", "linelist"])
@pytest.mark.parametrize("nnu", [2, 3, 257])
def test_slopes_bit_exact(m3d, oracle, kind, nnu):
    from dispatch_b200.optab import SampleOptab
    from oracle import optab
    tab = oc.table(kind, nnu=nnu)
    T = SampleOptab.from_dict(tab)
    for comp, name in ((0, "val"), (1, "scat")):
        for g, o in zip(T.slopes(comp), optab.slopes(tab, name)):
            np.testing.assert_array_equal(g, o)
    T.close()


@pytest.mark.parametrize("kind", ["background", "linelist"])
def test_sample_bit_exact(m3d, oracle, kind):
    from dispatch_b200.optab import SampleOptab
    from oracle import optab
    c = oc.cells()
    tab = oc.table(kind, nnu=400, cells_=c)
    q = np.sort(np.random.default_rng(4).uniform(3900.0, 9100.0, 150))   # beyond both ends too
    T = SampleOptab.from_dict(tab)
    b_g, s_g = T.interpolate(c["temp"], c["ne"], c["chi500"], q)
    b_o, s_o = optab.sample(tab, c["temp"], c["ne"], c["chi500"], q)
    np.testing.assert_array_equal(b_g, b_o)
    np.testing.assert_array_equal(s_g, s_o)
    assert b_o.max() > 0
    T.close()


@pytest.mark.parametrize("with_scat", [True, False])
@pytest.mark.parametrize("table_scat", [True, False])
def test_sample_ll_bit_exact(m3d, oracle, with_scat, table_scat):
    from dispatch_b200.optab import SampleOptab
    from oracle import optab
    c = oc.cells()
    tab = oc.table("linelist", nnu=500, scat=table_scat, cells_=c)
    q = np.linspace(4050.0, 8950.0, 200)
    vp = (c["vproj"] * 40.0).astype(np.float32)          # up to ~1e-3: several nodes of shift
    n = c["temp"].size
    rng = np.random.default_rng(5)
    base = [rng.random((n, q.size)).astype(np.float32) for _ in range(3)]
    out = {}
    T = SampleOptab.from_dict(tab)
    for name in ("g", "o"):
        x, e, s = (b.copy() for b in base)
        cs = s if with_scat else None
        if name == "g":
            T.interpolate_ll(c["temp"], c["ne"], c["chi500"], x, e, q, vp, cs)
        else:
            optab.sample_ll(tab, c["temp"], c["ne"], c["chi500"], vp, q, x, e, cs)
        out[name] = (x, e, s)
    for a, b in zip(out["g"], out["o"]):
        np.testing.assert_array_equal(a, b)
    assert not np.array_equal(out["o"][0], base[0])
    if not (with_scat and table_scat):
        np.testing.assert_array_equal(out["o"][2], base[2])
    T.close()


def test_device_tensors_and_checks(m3d, oracle):
    import torch
    from dispatch_b200.optab import SampleOptab
    from oracle import optab
    c = oc.cells(seed=3, nx=20, ny=20, nz=24)
    tab = oc.table("background", nnu=300, cells_=c)
    q = np.linspace(4100.0, 8900.0, 96)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    T = SampleOptab(dev(tab["lam"]), dev(tab["val"]), dev(tab["scat"]), tab["pca"])
    b, s = T.interpolate(dev(c["temp"]), dev(c["ne"]), dev(c["chi500"]), dev(q))
    torch.cuda.synchronize()
    b_o, s_o = optab.sample(tab, c["temp"], c["ne"], c["chi500"], q)
    np.testing.assert_array_equal(b.cpu().numpy(), b_o)
    np.testing.assert_array_equal(s.cpu().numpy(), s_o)
    x = torch.zeros_like(b)
    e = torch.zeros_like(b)
    T.interpolate_ll(dev(c["temp"]), dev(c["ne"]), dev(c["chi500"]), x, e, dev(q), dev(c["vproj"]))
    torch.cuda.synchronize()
    xo, eo = np.zeros_like(b_o), np.zeros_like(b_o)
    optab.sample_ll(tab, c["temp"], c["ne"], c["chi500"], c["vproj"], q, xo, eo)
    np.testing.assert_array_equal(x.cpu().numpy(), xo)
    T.close()
    bad = dict(tab)
    bad["lam"] = tab["lam"][::-1].copy()
    with pytest.raises(m3d.M3DError, match="ascend"):
        SampleOptab.from_dict(bad)
    one = {"lam": tab["lam"][:1], "val": tab["val"][..., :1].copy(), "scat": None, "pca": tab["pca"]}
    with pytest.raises(m3d.M3DError, match="two wavelengths"):
        SampleOptab.from_dict(one)
    ll = oc.table("linelist", nnu=50, scat=False, cells_=c)
    T2 = SampleOptab.from_dict(ll)
    with pytest.raises(m3d.M3DError, match="scattering component"):
        T2.interpolate(c["temp"], c["ne"], c["chi500"], q)
    T2.close()


def test_window_tables_bit_exact(m3d, oracle):
    """The tables as the reference builds them for a window: every background
    query on a node (the device's one-node collapse against the oracle's full
    one), the line-list queries shifted between the padded nodes."""
    from dispatch_b200 import synth
    from dispatch_b200.optab import SampleOptab
    from oracle import optab
    c = oc.cells(seed=5)
    q, bg, ll = synth.window_tables(3, c["temp"], c["ne"], c["vproj"], nf=96)
    T = SampleOptab.from_dict(bg)
    b_g, s_g = T.interpolate(c["temp"], c["ne"], c["chi500"], q)
    b_o, s_o = optab.sample(bg, c["temp"], c["ne"], c["chi500"], q)
    np.testing.assert_array_equal(b_g, b_o)
    np.testing.assert_array_equal(s_g, s_o)
    T.close()
    T = SampleOptab.from_dict(ll)
    n = c["temp"].size
    vp = c["vproj"].copy()
    vp[::7] = 0.0                                     # cells at rest query the nodes themselves
    out = {}
    for name in ("g", "o"):
        x, e, s = (np.zeros((n, q.size), np.float32) for _ in range(3))
        if name == "g":
            T.interpolate_ll(c["temp"], c["ne"], c["chi500"], x, e, q, vp, s)
        else:
            optab.sample_ll(ll, c["temp"], c["ne"], c["chi500"], vp, q, x, e, s)
        out[name] = (x, e, s)
    for a, b in zip(out["g"], out["o"]):
        np.testing.assert_array_equal(a, b)
    T.close()

"""Line lists with a per-line reach from a previous run (has_reach): select_lines
(linelist_mod.f90:1110-1142) and the branch of add_opacity_equi for lines centred
beyond the chunk -- the unfloored reference at the nearer end, no peak test, a
window capped by the reach (:844-854, 914-921).

CPU: the oracle's selection against a literal numpy statement of select_lines.
GPU: the line kernel (with its diagnostics, host and device pointers) and the
whole synthesis pass against the oracle, bit for bit."""
import numpy as np
import pytest

from tests.test_gpu_parity import _line_case


def _select_numpy(llam0, reach_in, active, llam, vmax):
    nf = llam.size
    hb1, hb2 = 0.5 * (llam[1] - llam[0]), 0.5 * (llam[-1] - llam[-2])
    blue = llam[0] - hb1 - float(vmax)
    red = llam[-1] + hb2 + float(vmax)
    rmax = float(reach_in.max())
    l0 = int(np.searchsorted(llam0, blue - rmax, "left"))       # first llam0 >= x
    l1 = int(np.searchsorted(llam0, red + rmax, "right")) - 1   # last llam0 <= x
    out = []
    for l in range(max(l0, 0), min(l1, llam0.size - 1) + 1):
        if active is not None and not active[l]:
            continue
        r = float(reach_in[l])
        if llam0[l] + r < blue or llam0[l] - r > red:
            continue
        out.append(l)
    return np.array(out, np.int32)


def test_select_lines_matches_numpy(oracle):
    sp, llam, xhat, cells, _ = _line_case(21, nline=300)
    rng = np.random.default_rng(2)
    sp = dict(sp)
    sp["reach_in"] = (10 ** rng.uniform(-6, -3.3, 300)).astype(np.float32)
    sp["active"] = (rng.random(300) < 0.9).astype(np.uint8)
    for vmax in (0.0, 3e-6, 1e-4):
        got = oracle.select_lines(sp, llam, vmax)
        ref = _select_numpy(sp["llam0"], sp["reach_in"], sp["active"], np.asarray(llam, np.float64), np.float32(vmax))
        assert np.array_equal(got, ref)
        assert 0 < got.size < 300


def _reach_case(oracle, seed):
    sp, llam, xhat, cells, dep = _line_case(seed, nline=200)
    lr = oracle.logref(xhat)
    # the reach of a first pass, shrunk for some lines so that the cap binds
    c, e = np.zeros_like(xhat), np.zeros_like(xhat)
    used, strength, reach = oracle.add_opacity_equi(sp, llam, c, e, xhat, lr, cells)
    rng = np.random.default_rng(seed)
    sp = dict(sp)
    sp["reach_in"] = (np.maximum(reach, 1e-7) * rng.choice([0.4, 1.0, 2.0], reach.size)).astype(np.float32)
    return sp, llam, xhat, lr, cells, dep


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
def test_line_opacity_reach_bit_exact(m3d, oracle, device):
    sp, llam, xhat, lr, cells, dep = _reach_case(oracle, 31)
    rng = np.random.default_rng(3)
    chi0 = (xhat * rng.uniform(0, 2, xhat.shape)).astype(np.float32)
    oc, oe = chi0.copy(), chi0.copy()
    ou, os_, orch = oracle.add_opacity_equi(sp, llam, oc, oe, xhat, lr, cells)
    if not device:
        gc, ge = chi0.copy(), chi0.copy()
        gu, gs, gr = m3d.line_opacity(sp, llam, gc, ge, xhat, lr, cells, diag=True)
    else:
        import torch
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        spd = {k: (d(v) if isinstance(v, np.ndarray) else v) for k, v in sp.items()}
        cd = {k: d(v) for k, v in cells.items()}
        gct, get = d(chi0), d(chi0)
        gu, gs, gr = m3d.line_opacity(spd, d(llam), gct, get, d(xhat), d(lr), cd, diag=True)
        gc, ge = gct.cpu().numpy(), get.cpu().numpy()
        gu, gs, gr = (x.cpu().numpy() if hasattr(x, "cpu") else x for x in (gu, gs, gr))
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gs, os_)
    np.testing.assert_array_equal(gr, orch)
    assert ou.sum() > 10


@pytest.mark.gpu
@pytest.mark.parametrize("nf,window", [(32, 5), (64, 2)])
def test_lte_synthesis_reach(m3d, oracle, nf, window):
    from dispatch_b200 import synth
    from oracle import pipeline as P
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=nf, window=window)
    rng = np.random.default_rng(7)
    n = atm["species"][0]["llam0"].size
    atm["species"][0]["reach_in"] = (10 ** rng.uniform(-6, -4, n)).astype(np.float32)
    ie, flux, itop = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    oie, oflux, oitop = P.lte_synthesis(atm, nu, llam, vec, wmu)
    np.testing.assert_array_equal(itop, oitop)
    np.testing.assert_allclose(flux, oflux, rtol=2e-6)
    # the reach changes the result against the list without it
    del atm["species"][0]["reach_in"]
    _, _, itop0 = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    assert not np.array_equal(itop0, itop)

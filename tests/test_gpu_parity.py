"""CUDA path against the oracle on the same seeded inputs, through the C ABI.

FP32 results must agree bit for bit: the kernels and the oracle evaluate the
reference's real(4) expressions in the same order (explicit fused multiply-adds
on both sides, no other contraction).  Window indices and line diagnostics are
integer or max-reductions and must agree exactly as well.  FP64 results agree to
rounding; reductions over the surface (ie, flux) to summation order.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand_t(n, seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.uniform(-2, 95, n), np.logspace(-8, 0, 200), -np.logspace(-8, 0.3, 200),
                           [0.0, 1.0, -1.0, 2.0, -2.0, 87.0, 88.0]]).astype(np.float32)


def test_k0_bit_exact(m3d, oracle):
    t = _rand_t(20000, 1)
    for which, fn in ((1, oracle.linear_weights), (2, oracle.parab_moments)):
        got = m3d.weights(which, t)
        exp = fn(t)
        for g, e in zip(got, exp):
            np.testing.assert_array_equal(g, e)
    E, u0 = m3d.weights(0, t)
    eE, eu0 = oracle.exp_neg(t)
    np.testing.assert_array_equal(E, eE)
    np.testing.assert_array_equal(u0, eu0)
    for g, e in zip(m3d.weights(5, t), oracle.bezier3_weights(t)):
        np.testing.assert_array_equal(g, e)
    x = np.linspace(-90, 90, 5001).astype(np.float32)
    np.testing.assert_array_equal(m3d.weights(3, x), oracle.exp4(x))
    x = np.float32(np.logspace(-40, 38, 5001))
    np.testing.assert_array_equal(m3d.weights(4, x), oracle.logf(x))


def test_k0_fp64(m3d, oracle):
    t = np.concatenate([np.logspace(-9, 2, 500), -np.logspace(-9, 0.3, 200)])
    for which, fn in ((1, oracle.linear_weights), (2, oracle.parab_moments)):
        for g, e in zip(m3d.weights(which, t, fp64=True), fn(t, fp64=True)):
            np.testing.assert_allclose(g, e, rtol=1e-14, atol=1e-300)


def test_qlg_tables_and_profile(m3d, oracle):
    tg, th = m3d.qlg_tables()
    otg, oth = oracle.qlg_tables()
    np.testing.assert_array_equal(tg, otg)
    np.testing.assert_array_equal(th, oth)
    rng = np.random.default_rng(2)
    n = 4000
    a = (10 ** rng.uniform(-4, 2, n)).astype(np.float32)
    q = rng.uniform(-1e-4, 1e-4, n).astype(np.float32)
    vpr = rng.uniform(-1e-5, 1e-5, n).astype(np.float32)
    idf = (10 ** rng.uniform(4, 5.5, n)).astype(np.float32)
    np.testing.assert_array_equal(m3d.qlg_bot_profile(a, q, vpr, idf), oracle.qlg_bot_profile(a, q, vpr, idf))


def _line_case(seed, nline=150, nf=300, ncell=48, nlevel=4, recipes=True):
    from dispatch_b200 import synth
    rng = np.random.default_rng(seed)
    raw = synth.random_linelist(rng, nline, 5000.0, 5006.0)
    temp = rng.uniform(3500, 9000, ncell).astype(np.float32)
    lt = rng.uniform(-5, 1, ncell)
    _, _, _, nH, ne = synth.grey_model(lt)
    sp = synth.species_arrays(raw, temp, 10 ** -4.5 * nH)
    if recipes:
        # damping constants already scaled by 1/(4 pi nu0), as the line list stores them
        # (line_types_mod.f90:36): gamma6 ~ 1e-8 cm^3/s, gamma4 ~ 1e-5 cm^3/s
        s4 = 1.0 / (4.0 * np.pi * (synth.HZ_TO_AA / raw["lam"]))
        sp["gw1"] = (10 ** rng.uniform(-9, -7.5, nline) * s4).astype(np.float32)
        sp["gw2"] = rng.uniform(0.3, 0.45, nline).astype(np.float32)
        sp["unsold"] = (rng.uniform(size=nline) < 0.5).astype(np.uint8)
        sp["gstk"] = (rng.choice([-1, 1], nline) * 10 ** rng.uniform(-6, -5, nline) * s4).astype(np.float32)
    sp["lev_i"] = rng.integers(0, nlevel + 1, nline).astype(np.int32)
    sp["lev_j"] = rng.integers(0, nlevel + 1, nline).astype(np.int32)
    cf = synth.cell_fields(temp, nH, ne)
    llam, nu = synth.frequency_grid(5000.5, 5005.5, nf)
    beta = np.exp(-6.626176e-27 * nu[None, :] / (1.380662e-16 * temp[:, None])).astype(np.float32)
    chi_c = (0.2 * 1e-7 * 10 ** rng.uniform(-2, 1, ncell)).astype(np.float32)
    xhat = (chi_c[:, None] * (1 + beta / (1 - beta))).astype(np.float32)
    cells = {"vproj": rng.uniform(-1e-5, 1e-5, ncell).astype(np.float32), "inv_df": sp["inv_df"],
             "vbar2": sp["vbar2"], "lnbase": sp["lnbase"], **cf}
    dep = rng.uniform(0.3, 3.0, (nlevel, ncell)).astype(np.float32)
    return sp, llam, xhat, cells, dep


@pytest.mark.parametrize("nlte", [False, True])
def test_line_opacity_bit_exact(m3d, oracle, nlte):
    sp, llam, xhat, cells, dep = _line_case(3 + nlte)
    lr = oracle.logref(xhat)
    ncell, nf = xhat.shape
    rng = np.random.default_rng(9)
    chi0 = (xhat * rng.uniform(0, 3, xhat.shape)).astype(np.float32)   # earlier species' opacity
    eta0 = (chi0 * 0.5).astype(np.float32)
    oc, oe = chi0.copy(), eta0.copy()
    ou, os_, orch = oracle.add_opacity_equi(sp, llam, oc, oe, xhat, lr, cells, dep_mem=dep, nlevel=dep.shape[0],
                                            do_nlte=nlte)
    gc, ge = chi0.copy(), eta0.copy()
    gu, gs, gr = m3d.line_opacity(sp, llam, gc, ge, xhat, lr, cells, dep_mem=dep, nlevel=dep.shape[0], do_nlte=nlte,
                                  diag=True)
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_array_equal(ge, oe)
    np.testing.assert_array_equal(gu, ou)
    np.testing.assert_array_equal(gs, os_)
    np.testing.assert_array_equal(gr, orch)
    assert ou.sum() > 10 and (gc != chi0).sum() > 100
    # without diagnostics the screened path deposits the same opacity
    hc, he = chi0.copy(), eta0.copy()
    m3d.line_opacity(sp, llam, hc, he, xhat, lr, cells, dep_mem=dep, nlevel=dep.shape[0], do_nlte=nlte)
    np.testing.assert_array_equal(hc, oc)
    np.testing.assert_array_equal(he, oe)


def test_line_opacity_floor_engages(m3d, oracle):
    """Strong lines over weak ones: the accumulated-opacity floor decides
    (linelist_mod.f90:857-869), and it decides identically."""
    sp, llam, xhat, cells, _ = _line_case(11, nline=300, recipes=False)
    sp["gpref"] = sp["gpref"] + np.float32(6.0)
    lr = oracle.logref(xhat)
    oc, oe = np.zeros_like(xhat), np.zeros_like(xhat)
    oracle.add_opacity_equi(sp, llam, oc, oe, xhat, lr, cells)
    assert (oc > 1e4 * xhat).any()
    gc, ge = np.zeros_like(xhat), np.zeros_like(xhat)
    m3d.line_opacity(sp, llam, gc, ge, xhat, lr, cells)
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_array_equal(ge, oe)


def test_background_and_units_bit_exact(m3d, oracle):
    rng = np.random.default_rng(4)
    nf, nc = 97, 33
    nu = np.linspace(2.9e14, 6.1e15, nf)
    temp = rng.uniform(2500, 30000, nc).astype(np.float32)
    b, B = m3d.lte_background(nu, temp)
    ob, oB = oracle.lte_background(nu, temp)
    np.testing.assert_array_equal(b, ob)
    np.testing.assert_array_equal(B, oB)
    w1 = rng.uniform(0.1, 2.0, (nc, nf)).astype(np.float32)
    w2 = (w1 * rng.uniform(0.2, 1.2, (nc, nf)) / b).astype(np.float32)
    w2[0, :5] = (w1[0, :5] / b[0, :5]).astype(np.float32)     # chi ~ 0: the maser floor
    g1, g2 = w1.copy(), w2.copy()
    n = m3d.work_to_transfer_units(g1, g2, b)
    o1, o2 = w1.copy(), w2.copy()
    on = oracle.work_to_transfer_units(o1, o2, ob)
    np.testing.assert_array_equal(g1, o1)
    np.testing.assert_array_equal(g2, o2)
    assert n == on


def _slab_case(seed, nf, nx, ny, nz, dtype, vec):
    rng = np.random.default_rng(seed)
    work = np.zeros((3, nz + 2, ny, nx, nf), dtype)
    work[0] = (10 ** rng.uniform(-9, -6, (nz + 2, ny, nx, nf))).astype(dtype)
    work[1] = rng.uniform(0.1, 3.0, (nz + 2, ny, nx, nf)).astype(dtype)
    work[2] = 0
    work[2, 0] = rng.uniform(0.1, 3.0, (ny, nx, nf)).astype(dtype)
    work[2, nz + 1] = rng.uniform(0.1, 3.0, (ny, nx, nf)).astype(dtype)
    # a few negative opacities (inverted populations) and near-zero ones
    m = rng.uniform(size=work[0].shape) < 0.01
    work[0][m] = -work[0][m] * 0.1
    chi500 = (10 ** rng.uniform(-8, -7, (nz, ny, nx))).astype(np.float32)
    chi500_up = (chi500 * rng.uniform(0.5, 2.0, chi500.shape)).astype(np.float32)
    chi500_up[0, 0, 0] = chi500[0, 0, 0] * np.float32(1.0004)
    g500 = (10 ** rng.uniform(-8, -7, (ny, nx))).astype(np.float32)
    eta_row = np.zeros((nz, ny, nx), np.int32)
    rows = rng.choice(eta_row.size, 6, replace=False)
    eta_row.ravel()[rows] = np.arange(1, 7)
    eta_mask = (rng.uniform(size=(6, nf)) < 0.4).astype(np.uint8)
    return work, chi500, chi500_up, g500, eta_row, eta_mask


SOLVERS = ["LINEAR", "LINEAR2", "QUADRATIC", "SHORT_LINEAR", "SHORT_LINEAR2"]


@pytest.mark.parametrize("solver", SOLVERS)
@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("dir", [1, -1])
def test_formal_solvers_bit_exact(m3d, oracle, solver, split, dir):
    if solver == "QUADRATIC" and split:
        pytest.skip("the quadratic solver has no split-rates form")
    nf, nx, ny, nz = 8, 12, 10, 6
    vec = np.array([0.31, -0.22, 0.0])
    vec[2] = dir * math.sqrt(1 - (vec[:2] ** 2).sum())
    ds = [1.2e7, 1.0e7, 0.8e7]
    work, c5, c5u, g5, er, em = _slab_case(17, nf, nx, ny, nz, np.float32, vec)
    s = getattr(oracle, solver)
    outs = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        w = work.copy()
        psi = np.zeros((nz, ny, nx, nf), np.float32)
        irem = np.zeros_like(psi) if split else None
        esc = np.zeros_like(psi) if split else None
        slab = mod.make_slab(nf, nx, ny, nz, dir, ds, vec, get_psi=True, split_rates=split)
        args = dict(psi=psi, irem=irem, escape=esc, chi500=c5, chi500_up=c5u, g500=g5, eta_row=er, eta_mask=em)
        if name == "o":
            oracle.formal_solve(s, slab, w, **args)
        else:
            m3d.formal_solve(getattr(m3d, solver), slab, w, **args)
        outs[name] = (w, psi, irem, esc)
    for a, b in zip(outs["g"], outs["o"]):
        if a is not None:
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("solver", SOLVERS)
def test_formal_solvers_fp64(m3d, oracle, solver):
    nf, nx, ny, nz = 6, 9, 8, 5
    vec = np.array([0.25, 0.4, math.sqrt(1 - 0.0625 - 0.16)])
    ds = [1.2e7, 1.0e7, 0.8e7]
    work, c5, c5u, g5, er, em = _slab_case(23, nf, nx, ny, nz, np.float64, vec)
    res = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        w = work.copy()
        psi = np.zeros((nz, ny, nx, nf), np.float64)
        irem, esc = np.zeros_like(psi), np.zeros_like(psi)
        slab = mod.make_slab(nf, nx, ny, nz, 1, ds, vec, get_psi=True, split_rates=solver != "QUADRATIC")
        args = dict(psi=psi, irem=irem, escape=esc, chi500=c5, chi500_up=c5u, g500=g5, eta_row=er, eta_mask=em)
        if name == "o":
            oracle.formal_solve(getattr(oracle, solver), slab, w, **args)
        else:
            m3d.formal_solve(getattr(m3d, solver), slab, w, **args)
        res[name] = (w, psi, irem, esc)
    for a, b in zip(res["g"], res["o"]):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-300)


def test_rotate_and_boundaries_bit_exact(m3d, oracle):
    nf, nx, ny, nz = 5, 11, 9, 7
    vec = np.array([0.5, -0.3, math.sqrt(1 - 0.34)])
    work, *_ = _slab_case(31, nf, nx, ny, nz, np.float32, vec)
    ds_code = (0.12, 0.1, 0.08)
    for b2p in (0.9, 3.1):
        wo, wg = work.copy(), work.copy()
        so = oracle.make_slab(nf, nx, ny, nz, 1, [1e7] * 3, vec)
        sg = m3d.make_slab(nf, nx, ny, nz, 1, [1e7] * 3, vec)
        oracle.rotate_array(so, wo, ds_code, b2p, (0.25, -0.5))
        m3d.rotate_array(sg, wg, ds_code, b2p, (0.25, -0.5))
        np.testing.assert_array_equal(wg, wo)
    rng = np.random.default_rng(5)
    mem = rng.uniform(0, 1, (3, ny, nx, nf)).astype(np.float32)
    r500 = rng.uniform(0.5, 2, (ny, nx)).astype(np.float32)
    gt = rng.uniform(5000, 12000, (ny, nx)).astype(np.float32)
    nu = np.linspace(5e14, 7e14, nf)
    for mode in (m3d.BND_MEM, m3d.BND_ZERO, m3d.BND_PCHIP, m3d.BND_LTE):
        for dir in (1, -1):
            wo, wg = work.copy(), work.copy()
            so = oracle.make_slab(nf, nx, ny, nz, dir, [1e7] * 3, vec)
            sg = m3d.make_slab(nf, nx, ny, nz, dir, [1e7] * 3, vec)
            omode = {m3d.BND_MEM: oracle.BND_NONE, m3d.BND_ZERO: oracle.BND_ZERO, m3d.BND_PCHIP: oracle.BND_PCHIP,
                     m3d.BND_LTE: oracle.BND_LTE}[mode]
            oracle.upstream_boundary(so, wo, omode, mem=mem, ds3_code=np.float32(0.08), ghost_r500=r500,
                                     ghost_temp=gt, nu=nu)
            m3d.upstream_boundary(sg, wg, mode, mem=mem, ds3_code=0.08, ghost_r500=r500, ghost_temp=gt, nu=nu)
            np.testing.assert_array_equal(wg, wo)


def test_integrate_intensity(m3d, oracle):
    rng = np.random.default_rng(8)
    I = rng.uniform(0, 1, 5000).astype(np.float32)
    P = rng.uniform(0, 1, 5000).astype(np.float32)
    J0 = rng.uniform(0, 1, 5000).astype(np.float32)
    PJ0 = rng.uniform(0, 1, 5000).astype(np.float32)
    gJ, gP = J0.copy(), PJ0.copy()
    m3d.integrate_intensity(0.0833, I, P, gJ, gP)
    oJ, oP = J0.copy(), PJ0.copy()
    oracle.integrate_intensity(0.0833, I, P, oJ, oP)
    np.testing.assert_array_equal(gJ, oJ)
    np.testing.assert_array_equal(gP, oP)


@pytest.mark.parametrize("kind,nf,window", [("mini", 64, 2), ("c0", 256, 31), ("mini", 32, 5), ("c0", 32, 200)])
def test_lte_synthesis_matches_oracle(m3d, oracle, kind, nf, window):
    from dispatch_b200 import synth
    from oracle import pipeline as P
    atm, nu, llam, vec, wmu = synth.lte_config(kind, nf=nf, window=window)
    n0 = m3d.launch_count()
    ie, flux, itop = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    assert m3d.launch_count() > n0
    oie, oflux, oitop = P.lte_synthesis(atm, nu, llam, vec, wmu)
    np.testing.assert_array_equal(itop, oitop)
    np.testing.assert_allclose(ie, oie, rtol=2e-6)
    np.testing.assert_allclose(flux, oflux, rtol=2e-6)
    # the plain FP64 path against the FP64 oracle, and the FP32 error it measures
    ie64, flux64, itop64 = m3d.lte_synthesis(atm, nu, llam, vec, wmu, fp64=True, return_itop=True)
    oie64, oflux64, oitop64 = P.lte_synthesis(atm, nu, llam, vec, wmu, fp64=True)
    np.testing.assert_allclose(itop64, oitop64, rtol=1e-11)
    assert np.max(np.abs(flux - flux64) / flux64) <= 1e-4


def test_lte_synthesis_device_pointers_match_host(m3d):
    import torch
    from dispatch_b200 import synth
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=48, window=3)
    ie_h, flux_h, itop_h = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)

    def dev(x):
        return torch.from_numpy(np.ascontiguousarray(x)).cuda()

    datm = {k: (dev(v) if isinstance(v, np.ndarray) and k != "slab_nz" else v) for k, v in atm.items()}
    datm["species"] = [{k: dev(v) for k, v in sp.items()} for sp in atm["species"]]
    torch.cuda.synchronize()
    ie_d, flux_d, itop_d = m3d.lte_synthesis(datm, dev(nu), dev(llam), vec, wmu, return_itop=True, device=True)
    m3d.synchronize()
    np.testing.assert_array_equal(itop_d.cpu().numpy(), itop_h)
    np.testing.assert_array_equal(ie_d.cpu().numpy(), ie_h)
    np.testing.assert_array_equal(flux_d.cpu().numpy(), flux_h)


def test_full_size_window_properties(m3d):
    """The 240^3, 10-slab cube of the 3D LTE configuration, one window, two rays:
    sizes where every launch needs many waves of blocks.  Size-independent
    properties: the FP32 path is within 1e-4 of the plain FP64 path, intensities
    are positive and finite, and lines only remove flux from the continuum."""
    from dispatch_b200 import synth
    cube = synth.cube_atmosphere(1, 240, 240, 240)
    atm, nu, llam, vec, wmu = synth.lte_config("c1", nf=32, window=62, cube=cube)
    vec, wmu = vec[[0, 12]], wmu[[0, 12]]
    ie, flux, itop = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    ie64, flux64, _ = m3d.lte_synthesis(atm, nu, llam, vec, wmu, fp64=True)
    assert np.all(np.isfinite(itop)) and np.all(itop > 0)
    assert np.max(np.abs(flux - flux64) / flux64) <= 1e-4
    assert np.max(np.abs(ie - ie64) / ie64) <= 1e-4
    cont = dict(atm)
    cont["species"] = []
    _, fc, _ = m3d.lte_synthesis(cont, nu, llam, vec, wmu)
    assert np.all(flux <= fc * (1 + 1e-6))
    assert np.min(flux / fc) < 0.9


@pytest.mark.parametrize("nlte", [False, True])
def test_line_opacity_scattering_split_bit_exact(m3d, oracle, nlte):
    """line_scattering (linelist_mod.f90:933-939): an LTE line adds (1-eps) of its
    profile to chi_scat; a departure-carrying line adds none."""
    sp, llam, xhat, cells, dep = _line_case(21 + nlte)
    lr = oracle.logref(xhat)
    rng = np.random.default_rng(4)
    ome = rng.uniform(0.0, 1.0, xhat.shape).astype(np.float32)
    chi0 = (xhat * rng.uniform(0, 2, xhat.shape)).astype(np.float32)
    out = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        c, e, cs = chi0.copy(), (chi0 * 0.5).astype(np.float32), np.zeros_like(chi0)
        if name == "o":
            oracle.add_opacity_equi(sp, llam, c, e, xhat, lr, cells, dep_mem=dep, nlevel=dep.shape[0], do_nlte=nlte,
                                    one_m_eps=ome, chi_scat=cs)
        else:
            m3d.line_opacity(sp, llam, c, e, xhat, lr, cells, dep_mem=dep, nlevel=dep.shape[0], do_nlte=nlte,
                             one_m_eps=ome, chi_scat=cs)
        out[name] = (c, e, cs)
    for a, b in zip(out["g"], out["o"]):
        np.testing.assert_array_equal(a, b)
    assert out["o"][2].max() > 0


def test_chi_scat_units(m3d):
    """chi_scat * (1 - beta) in real(4), as add_linelist_opacities converts it."""
    rng = np.random.default_rng(8)
    cs = rng.uniform(0, 1e-6, (50, 37)).astype(np.float32)
    beta = rng.uniform(0, 1, cs.shape).astype(np.float32)
    exp = (cs * (np.float32(1.0) - beta)).astype(np.float32)
    got = cs.copy()
    m3d.rt.chi_scat_units(got, beta)
    np.testing.assert_array_equal(got, exp)


def test_save5_from_device_buffers(m3d, tmp_path):
    """The output files written straight from device tensors equal those from host buffers."""
    import os

    import torch
    from dispatch_b200 import output
    a = np.random.default_rng(2).random((2, 1, 1, 3, 40)).astype(np.float32)
    output.save5(str(tmp_path / "h"), "J", (3, 1, 7), a)
    output.save5(str(tmp_path / "d"), "J", (3, 1, 7), torch.from_numpy(a).cuda())
    for f in ("J_003001007.bin", "J_meta.txt"):
        assert open(os.path.join(str(tmp_path / "h"), "save", f), "rb").read() == \
            open(os.path.join(str(tmp_path / "d"), "save", f), "rb").read()

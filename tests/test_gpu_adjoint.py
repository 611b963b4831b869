"""The hand-written adjoint of the LTE pass (m3d_lte_synthesis_adjoint) and the
differentiable front end over it (dispatch_b200.autodiff), against central finite
differences.

The case is the differentiable configuration at a small size: a 12 x 12 x 32 seeded
cube in two slabs of 16 planes, ten species of 20 lines each in 6000-6050 A, one
window of 32 of the 8000 frequencies, 13 Lobatto rays.  The loss is a seeded positive
weighting of the window's flux.  The finite differences are taken on the plain FP64
path, so they carry no FP32 rounding noise; the adjoint is the derivative of the FP32
pass, so they agree to the FP32 path's own accuracy plus the effect of QLG-bot's
nearest-node profile (the adjoint differentiates the continuous member the table
samples).  Steps: 1e-3 dex for log gf and abundances, 1 K for temperatures, 1e-3
relative for the continuum; tolerances as stated in each test."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LN10 = math.log(10.0)


@pytest.fixture(scope="module")
def case():
    from dispatch_b200 import synth
    atm, nu, llam, vec, wmu, raw = synth.lte_config_c4(size=(12, 12, 32), nline_per_species=20, window=100)
    rng = np.random.default_rng(11)
    wts = rng.uniform(0.5, 1.5, nu.size)
    return atm, nu, llam, vec, wmu, raw, wts


def _loss(m3d, atm, nu, llam, vec, wmu, wts):
    """The weighted flux of the plain FP64 path, formed in double from its float64
    emergent intensities (save_intensity's sum, rt_patch_mod.f90:4151-4208), since the
    pass returns ie and flux rounded to float32."""
    _, _, itop = m3d.lte_synthesis(atm, nu, llam, vec, wmu, fp64=True, return_itop=True)
    conv = 2.0 * 6.626176e-27 / (2.99792458e10 ** 3 * 1e8)
    ie = conv * nu ** 5 * itop.reshape(itop.shape[0], -1, nu.size).mean(axis=1)
    flux = (2.0 * 3.14159265359 * wmu)[:, None] * ie
    return float(np.dot(wts, flux.sum(axis=0)))


def _with(atm, **changes):
    out = dict(atm)
    out["species"] = [dict(sp) for sp in atm["species"]]
    for k, v in changes.items():
        if k == "species":
            for i, sp in v.items():
                out["species"][i].update(sp)
        else:
            out[k] = v
    return out


@pytest.fixture(scope="module")
def grads(m3d, case):
    atm, nu, llam, vec, wmu, raw, wts = case
    return m3d.lte_synthesis_adjoint(atm, nu, llam, vec, wmu, wts.astype(np.float32))


def test_gradient_log_gf(m3d, case, grads):
    """dL/dgpref of the five most sensitive lines, within 2 % of the differences."""
    atm, nu, llam, vec, wmu, raw, wts = case
    g = grads["gpref"]
    assert np.all(np.isfinite(g)) and np.abs(g).max() > 0
    h = 1e-3 * LN10
    sizes = [len(sp["llam0"]) for sp in atm["species"]]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for j in np.argsort(-np.abs(g))[:5]:
        k = int(np.searchsorted(offs, j, side="right") - 1)
        i = j - offs[k]
        vals = []
        for s in (+1, -1):
            gp = atm["species"][k]["gpref"].copy()
            gp[i] = np.float32(gp[i] + s * h)
            vals.append((_loss(m3d, _with(atm, species={k: {"gpref": gp}}), nu, llam, vec, wmu, wts), gp[i]))
        fd = (vals[0][0] - vals[1][0]) / (float(vals[0][1]) - float(vals[1][1]))
        assert abs(g[j] - fd) <= 2e-2 * abs(fd), (j, g[j], fd)


def test_gradient_abundances(m3d, case, grads):
    """dL/dA_X = ln 10 sum_cells dL/dlnbase_X for the three most sensitive species,
    within 2 %."""
    atm, nu, llam, vec, wmu, raw, wts = case
    gA = LN10 * grads["lnbase"].astype(np.float64).sum(axis=1)
    h = 1e-3
    for k in np.argsort(-np.abs(gA))[:3]:
        vals = []
        for s in (+1, -1):
            lnb = (atm["species"][k]["lnbase"].astype(np.float64) + s * h * LN10).astype(np.float32)
            vals.append(_loss(m3d, _with(atm, species={int(k): {"lnbase": lnb}}), nu, llam, vec, wmu, wts))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(gA[k] - fd) <= 2e-2 * abs(fd), (k, gA[k], fd)


def test_gradient_continuum(m3d, case, grads):
    """dL/dchi_c of four cells (the sweep, its rotation and the transfer units),
    within 1 %."""
    atm, nu, llam, vec, wmu, raw, wts = case
    g = grads["chi_c"]
    for c in np.argsort(-np.abs(g * atm["chi_c"]))[:4]:
        vals, xs = [], []
        for s in (+1, -1):
            cc = atm["chi_c"].copy()
            cc[c] = np.float32(cc[c] * (1 + s * 1e-3))
            xs.append(float(cc[c]))
            vals.append(_loss(m3d, _with(atm, chi_c=cc), nu, llam, vec, wmu, wts))
        fd = (vals[0] - vals[1]) / (xs[0] - xs[1])
        assert abs(g[c] - fd) <= 1e-2 * abs(fd), (c, g[c], fd)


def test_gradient_temperature(m3d, case, grads):
    """dL/dT of four cells: the background's direct term plus the Doppler factor,
    lnbase and e_kT through their formulas, within 5 % (a 1 K step moves profile
    points across QLG table nodes, which the continuous derivative smooths over)."""
    from dispatch_b200 import synth
    atm, nu, llam, vec, wmu, raw, wts = case
    temp = atm["temp"].astype(np.float64)
    const = 2.0 * synth.BK / synth.UU
    vmic2 = (1e5) ** 2
    dT = grads["temp"].astype(np.float64) + grads["e_kT"] * (-atm["e_kT"].astype(np.float64) / temp)
    for k, a in enumerate(raw["awgt"]):
        dop = const * temp / a + vmic2
        didf = -0.5 * atm["species"][k]["inv_df"].astype(np.float64) * (const / a) / dop
        dT = dT + grads["inv_df"][k] * didf + grads["lnbase"][k] * didf / atm["species"][k]["inv_df"]

    def fields(T):
        out = {"temp": T.astype(np.float32)}
        out.update({k: v for k, v in synth.cell_fields(T.astype(np.float32), raw["nH"],
                                                       atm["ne"]).items() if k in ("e_kT",)})
        sp = {}
        for k, a in enumerate(raw["awgt"]):
            n_x = 10.0 ** (raw["abund"][k] - 12.0) * raw["nH"]
            full = synth.species_arrays(raw["lines"][k], T.astype(np.float32), n_x, awgt=a)
            sp[k] = {"inv_df": full["inv_df"], "lnbase": full["lnbase"]}
        return out, sp

    for c in np.argsort(-np.abs(dT))[:4]:
        vals = []
        for s in (+1, -1):
            T = temp.copy()
            T[c] += s * 1.0
            f, sp = fields(T)
            vals.append(_loss(m3d, _with(atm, species=sp, **f), nu, llam, vec, wmu, wts))
        fd = (vals[0] - vals[1]) / 2.0
        assert abs(dT[c] - fd) <= 5e-2 * abs(fd), (c, dT[c], fd)


def test_autograd_front_end(m3d, case, grads):
    """LteSpectrum.flux(...).backward() gives the library adjoint's gradients composed
    through the fields' formulas (abundances and log gf to FP32 rounding), and its
    log gf gradient agrees with a finite difference of the FP32 front end itself."""
    import torch
    from dispatch_b200.autodiff import LteSpectrum
    atm, nu, llam, vec, wmu, raw, wts = case
    spec = LteSpectrum(atm, raw, vec, wmu)
    T = torch.tensor(raw["temp"], dtype=torch.float32, device="cuda", requires_grad=True)
    A = torch.tensor(raw["abund"], dtype=torch.float64, device="cuda", requires_grad=True)
    gf = torch.tensor(np.concatenate([r["loggf"] for r in raw["lines"]]), dtype=torch.float64, device="cuda",
                      requires_grad=True)
    w = torch.tensor(wts, dtype=torch.float32, device="cuda")
    loss = (spec.flux(T, A, gf, [100]) * w).sum()
    loss.backward()
    gA = A.grad.cpu().numpy()
    np.testing.assert_allclose(gA, LN10 * grads["lnbase"].astype(np.float64).sum(axis=1), rtol=1e-4,
                               atol=1e-6 * np.abs(gA).max())
    np.testing.assert_allclose(gf.grad.cpu().numpy(), LN10 * grads["gpref"], rtol=1e-4,
                               atol=1e-6 * np.abs(gf.grad.cpu().numpy()).max())
    assert torch.isfinite(T.grad).all()
    j = int(torch.argmax(torch.abs(gf.grad)))
    h = 1e-2
    with torch.no_grad():
        lp, lm = [], []
        for s, acc in ((+1, lp), (-1, lm)):
            g2 = gf.detach().clone()
            g2[j] += s * h
            acc.append(float((spec.flux(T.detach(), A.detach(), g2, [100]) * w).sum()))
    fd = (lp[0] - lm[0]) / (2 * h)
    assert abs(float(gf.grad[j]) - fd) <= 5e-2 * abs(fd)

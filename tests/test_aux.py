"""The auxiliary steps around the solvers: update_eta_mask's flags
(rt_patch_mod.f90:3671-3807), compute_lte_populations with the level partition
function (atom_mod.f90:1041-1150) and add_particle_opacity's per-cell fields
(ion_mod.f90:198-221, linelist_mod.f90:1023-1042).

CPU: the oracle's flag geometry on a single fired point.  GPU: the kernels against
the oracle -- the flags and the thermal fields bit for bit, the populations and
lnbase within the ulps of the device's exp/log (stated per test)."""
import numpy as np
import pytest

from dispatch_b200 import synth


@pytest.fixture(scope="module")
def ax(oracle):
    from oracle import aux
    return aux


def _slab_arrays(nf, nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    work = np.zeros((3, nz + 2, ny, nx, nf), np.float32)
    work[0] = rng.uniform(1e-3, 1.0, work[0].shape)
    work[1] = rng.uniform(0.1, 10.0, work[1].shape)
    neg = rng.random(work[0].shape) < 0.01
    work[0][neg] *= -1.0
    beta = rng.uniform(0.0, 1.0, (nz, ny, nx, nf)).astype(np.float32)
    return work, beta


def test_eta_oracle_geometry(ax):
    nf, nx, ny, nz = 2, 9, 8, 5
    work, beta = _slab_arrays(nf, nx, ny, nz, 0)
    work[0] = np.abs(work[0])
    work[0, 3, 4, 2, 1] = -1.0          # one fired point: plane z = 3 (1-based), y = 4, x = 2, f = 1
    src = np.zeros(beta.shape, np.uint8)
    mask = np.zeros(beta.shape, np.uint8)
    ax.update_eta_mask(work, beta, src, None, mask, dir=1, rx=1, ry=2, ghost=False)
    assert src.sum() == 1 and src[2, 4, 2, 1] == 1
    box = np.zeros((nz, ny, nx), bool)
    for z in (2, 3):
        for y in range(2, 7):
            for x in range(1, 4):
                box[z, y, x] = True
    assert np.array_equal(mask[..., 1].astype(bool), box) and mask[..., 0].sum() == 0
    # the flags only grow, and an old source adds nothing new
    m0 = mask.copy()
    ax.update_eta_mask(work, beta, src, None, mask, dir=1, rx=1, ry=2, ghost=False)
    assert np.array_equal(mask, m0)


@pytest.mark.gpu
@pytest.mark.parametrize("dir,ghost", [(1, True), (-1, True), (1, False)])
def test_eta_mask_gpu(m3d, ax, dir, ghost):
    nf, nx, ny, nz = 8, 10, 9, 7
    vec = (0.3, -0.2, 0.93) if dir > 0 else (0.3, -0.2, -0.93)
    slab = m3d.make_slab(nf, nx, ny, nz, dir, (1.0, 1.0, 1.0), vec)
    rx, ry = m3d.rt.eta_spread([vec], (1.0, 1.0, 1.0))
    out = []
    for impl in ("oracle", "gpu"):
        src = np.zeros((nz, ny, nx, nf), np.uint8)
        mask = np.zeros_like(src)
        gsrc = np.zeros((ny, nx, nf), np.uint8) if ghost else None
        for it in range(3):
            work, beta = _slab_arrays(nf, nx, ny, nz, 10 + it)
            if impl == "oracle":
                ax.update_eta_mask(work, beta, src, gsrc, mask, dir, rx, ry, ghost)
            else:
                m3d.rt.update_eta_mask(slab, work, beta, src, mask, rx, ry, eta_gsrc=gsrc)
        out.append((src, mask, gsrc))
    (so, mo, go), (sg, mg, gg) = out
    assert np.array_equal(sg, so) and np.array_equal(mg, mo)
    assert mo.sum() > so.sum() > 0
    if ghost:
        assert np.array_equal(gg, go)


@pytest.mark.gpu
def test_lte_populations_gpu(m3d, ax):
    atom, inp = synth.se_config("small", ncell=4096)
    temp = inp["temp"].astype(np.float32)
    lsaha = np.log(2.0 * (2.0 * np.pi * synth.EM * synth.BK * inp["temp"] / synth.HH**2) ** 1.5
                   / inp["ne"]).astype(np.float32)
    dxi = np.full(temp.size, 1e-3, np.float32)
    totn = inp["totn"].copy()
    ns_o, tot_o = ax.lte_populations(atom["g"], atom["ev"], atom["ion"], temp, lsaha, dxi, totn)
    ns_g = m3d.rt.lte_populations(atom, temp, lsaha, totn, dxi=dxi)
    np.testing.assert_allclose(ns_g, ns_o, rtol=1e-13, atol=0)    # device exp/log
    np.testing.assert_allclose(totn, tot_o, rtol=1e-13)
    np.testing.assert_allclose(ns_g.sum(axis=0), totn, rtol=1e-14)


@pytest.mark.gpu
def test_particle_fields_gpu(m3d, ax):
    rng = np.random.default_rng(4)
    temp = rng.uniform(3000, 12000, 5000).astype(np.float32)
    n = np.exp(rng.uniform(0, 30, 5000))
    n[:3] = 0.0
    part = rng.uniform(1, 4, 5000)
    for vmic, frac, scale in ((1.0, 1.0, 0.0), (0.0, 0.3, 2.5)):
        io, vo, lo = ax.particle_fields(55.847, vmic, frac, scale, temp, n, part)
        ig, vg, lg = m3d.rt.particle_fields(55.847, vmic, frac, temp, n, part, population_scale=scale)
        assert np.array_equal(ig, io) and np.array_equal(vg, vo)
        np.testing.assert_allclose(lg, lo, rtol=0, atol=4 * np.spacing(np.abs(lo)).max())   # log / logf ulps


@pytest.mark.gpu
@pytest.mark.parametrize("jmode,precond,valid", [(1, False, False), (2, False, False), (0, False, False),
                                                   (0, True, False), (0, True, True)])
def test_lte_emission_gpu(m3d, jmode, precond, valid):
    from oracle import nlte as onl
    rng = np.random.default_rng(jmode + 3 * precond + 7 * valid)
    shape = (500, 64)
    chi = rng.uniform(1e-9, 1e-6, shape).astype(np.float32)
    sigma = (chi * rng.uniform(0, 3, shape)).astype(np.float32)
    beta = rng.uniform(1e-6, 0.9, shape).astype(np.float32)
    Bnu = (beta / (1 - beta)).astype(np.float32)
    J = (Bnu * rng.uniform(0.2, 1.5, shape)).astype(np.float32)
    PsiJ = (rng.uniform(0, 2, shape) / chi).astype(np.float32) if precond else None
    Jali0 = (J * rng.uniform(0.5, 1.5, shape)).astype(np.float32)
    ja_o, ja_g = Jali0.copy(), Jali0.copy()
    xo, eo, do, no = onl.lte_emission(chi, sigma, Bnu, beta, J if jmode == 0 else None, jmode, PsiJ,
                                      ja_o if precond else None, valid, 0.9)
    xg, eg, dg, ng = m3d.rt.lte_emission(chi, Bnu, beta, sigma=sigma, Jnu=J if jmode == 0 else None,
                                         jnu_init=jmode, PsiJ=PsiJ, Jali=ja_g if precond else None,
                                         jali_valid=valid, scat_op_max=0.9)
    for a, b in ((xg, xo), (eg, eo), (dg, do), (ja_g, ja_o)):
        assert np.array_equal(a, b)
    assert ng == no
    if precond:
        assert no > 0 or not np.array_equal(ja_o, Jali0)

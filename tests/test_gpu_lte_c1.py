"""The LTE pass at the shape of the 3D LTE configuration, against the oracle.

A 48^3 cube built as the configuration's 240^3 one (same seeded fields, 10 depth
slabs, the same 500-line list in 5000-5020 A, 4000 frequencies in windows of 32,
all 13 Lobatto rays), three windows: both band edges and the middle.  The opacity
kernel chooses its window forms and reciprocal per warp by vote, so these cases
exercise those votes on the configuration's own line list.

* Transfer units (m3d_lte_transfer_units): every ray and window, bit for bit on a
  seeded sample of cells (the oracle's line loop is per cell; the bottom and top
  planes are always in the sample).
* The sweep: the oracle's column sweep run on the device's transfer units of the
  whole cube gives the device's emergent plane bit for bit, for every ray.
* The plain FP64 path against the FP64 oracle (1e-11), and the FP32 error
  against it for each output (chi, S, I_top, ie, flux)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WINDOWS = (0, 62, 124)


@pytest.fixture(scope="module")
def c1_48():
    from dispatch_b200 import synth
    cube = synth.cube_atmosphere(1, 48, 48, 48)
    out = {}
    for w in WINDOWS:
        out[w] = synth.lte_config("c1", nf=32, window=w, size=48, cube=cube)
    return out


def _sample_atm(atm, cells):
    sub = {"nx": cells.size, "ny": 1, "nz": 1, "slab_nz": [1]}
    for k in ("temp", "chi_c", "vx", "vy", "vz", "e_kT", "ne", "tothi", "stark_pe"):
        sub[k] = np.ascontiguousarray(atm[k][cells])
    sub["species"] = [{k: (np.ascontiguousarray(v[cells]) if k in ("inv_df", "vbar2", "lnbase") else v)
                       for k, v in sp.items()} for sp in atm["species"]]
    for k in ("tol", "maser_chi_floor"):
        if k in atm:
            sub[k] = atm[k]
    return sub


def _cells(atm, n=384, seed=5):
    nxy = atm["nx"] * atm["ny"]
    ncell = nxy * atm["nz"]
    rng = np.random.default_rng(seed)
    pick = rng.choice(ncell, n, replace=False)
    edge = np.concatenate([rng.choice(nxy, 32, replace=False), ncell - nxy + rng.choice(nxy, 32, replace=False)])
    return np.unique(np.concatenate([pick, edge]))


@pytest.mark.parametrize("w", WINDOWS)
def test_c1_transfer_units_and_sweep_bit_exact(m3d, oracle, c1_48, w):
    from oracle import pipeline as P
    atm, nu, llam, vec, wmu = c1_48[w]
    assert len(atm["species"][0]["llam0"]) == 500 and vec.shape[0] == 13
    cells = _cells(atm)
    sub = _sample_atm(atm, cells)
    _, _, itop = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    for r in range(vec.shape[0]):
        chi, S = m3d.lte_transfer_units(atm, nu, llam, vec[r])
        ochi, oS = P.transfer_units(sub, nu, llam, vec[r])
        np.testing.assert_array_equal(chi[cells], ochi, err_msg=f"chi, ray {r}, window {w}")
        np.testing.assert_array_equal(S[cells], oS, err_msg=f"S, ray {r}, window {w}")
        otop = P.column_sweep(atm, chi, S, vec[r])
        np.testing.assert_array_equal(itop[r], otop, err_msg=f"I_top, ray {r}, window {w}")


def test_transfer_units_mini_bit_exact_and_fp64(m3d, oracle):
    from dispatch_b200 import synth
    from oracle import pipeline as P
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=32, window=5)
    for r in (0, 5, 12):
        chi, S = m3d.lte_transfer_units(atm, nu, llam, vec[r])
        ochi, oS = P.transfer_units(atm, nu, llam, vec[r])
        np.testing.assert_array_equal(chi, ochi)
        np.testing.assert_array_equal(S, oS)
        c64, s64 = m3d.lte_transfer_units(atm, nu, llam, vec[r], fp64=True)
        oc64, os64 = P.transfer_units(atm, nu, llam, vec[r], fp64=True)
        np.testing.assert_allclose(c64, oc64, rtol=1e-11, atol=0)
        np.testing.assert_allclose(s64, os64, rtol=1e-11, atol=0)
    # windows of other widths take the FP64 kernel's general form
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=48, window=3)
    c64, s64 = m3d.lte_transfer_units(atm, nu, llam, vec[3], fp64=True)
    oc64, os64 = P.transfer_units(atm, nu, llam, vec[3], fp64=True)
    np.testing.assert_allclose(c64, oc64, rtol=1e-11, atol=0)
    np.testing.assert_allclose(s64, os64, rtol=1e-11, atol=0)


def test_c1_fp64_path_and_fp32_error(m3d, oracle, c1_48):
    """The plain FP64 path on the middle window against the FP64 oracle on the
    sampled cells, and the FP32 path's error against the FP64 path for each output.
    Bounds: flux and ie within 1e-4 (the configuration's requirement); chi, S and
    I_top: median within 1e-6 -- single points can differ by a table node, since
    QLG-bot snaps to the nearest of its nodes and FP32 and FP64 can round a point
    to different nodes (a jump of up to ~2e-3 in that point's line profile)."""
    from oracle import pipeline as P
    atm, nu, llam, vec, wmu = c1_48[62]
    cells = _cells(atm, n=128)
    sub = _sample_atm(atm, cells)
    for r in (0, 7):
        c64, s64 = m3d.lte_transfer_units(atm, nu, llam, vec[r], fp64=True)
        oc64, os64 = P.transfer_units(sub, nu, llam, vec[r], fp64=True)
        np.testing.assert_allclose(c64[cells], oc64, rtol=1e-11, atol=0)
        np.testing.assert_allclose(s64[cells], os64, rtol=1e-11, atol=0)
        c32, s32 = m3d.lte_transfer_units(atm, nu, llam, vec[r])
        ec = np.abs(c32 - c64) / np.abs(c64)
        es = np.abs(s32 - s64) / np.abs(s64)
        assert np.median(ec) < 1e-6 and np.median(es) < 1e-6
        assert np.max(ec) < 5e-3 and np.max(es) < 5e-3
    ie, flux, it32 = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    ie64, flux64, it64 = m3d.lte_synthesis(atm, nu, llam, vec, wmu, fp64=True, return_itop=True)
    assert np.max(np.abs(flux - flux64) / flux64) <= 1e-4
    assert np.max(np.abs(ie - ie64) / ie64) <= 1e-4
    ei = np.abs(it32 - it64) / np.abs(it64)
    assert np.median(ei) < 1e-6 and np.max(ei) < 5e-3

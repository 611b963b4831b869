"""m3d_lte_synthesis_windows: a batch of windows of 32 frequencies in one call equals
one m3d_lte_synthesis call per window bit for bit -- ie, flux and the emergent
planes of every ray, FP32 and the plain FP64 path -- on the 1D configuration (80
depths, 2000 lines: the case the batch is for) and on the small 3D cube (several
columns and slabs: the rows of the batch are the sweep's frequencies), with host and
device buffers; and one batched window against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(kind, w0, nwin):
    from dispatch_b200 import synth
    atm, nu, llam, vec, wmu = synth.lte_config(kind)
    sl = slice(32 * w0, 32 * (w0 + nwin))
    return atm, nu[sl].reshape(nwin, 32).copy(), llam[sl].reshape(nwin, 32).copy(), vec, wmu


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("kind,w0,nwin", [("c0", 100, 12), ("mini", 2, 5)])
def test_window_batch_equals_single_windows(m3d, kind, w0, nwin, fp64):
    atm, nu, llam, vec, wmu = _batch(kind, w0, nwin)
    ie, flux, itop = m3d.lte_synthesis_windows(atm, nu, llam, vec, wmu, fp64=fp64, return_itop=True)
    assert ie.shape == (wmu.size, 32 * nwin) and flux.shape == (32 * nwin,)
    for w in range(nwin):
        ie1, flux1, itop1 = m3d.lte_synthesis(atm, nu[w], llam[w], vec, wmu, fp64=fp64, return_itop=True)
        sl = slice(32 * w, 32 * (w + 1))
        np.testing.assert_array_equal(itop[..., sl], itop1, err_msg=f"window {w}")
        np.testing.assert_array_equal(ie[:, sl], ie1, err_msg=f"window {w}")
        np.testing.assert_array_equal(flux[sl], flux1, err_msg=f"window {w}")


def test_window_batch_device_pointers_and_oracle(m3d):
    import torch
    from oracle import pipeline as P
    atm, nu, llam, vec, wmu = _batch("c0", 400, 40)
    ie_h, flux_h, itop_h = m3d.lte_synthesis_windows(atm, nu, llam, vec, wmu, return_itop=True)

    def dev(x):
        return torch.from_numpy(np.ascontiguousarray(x)).cuda()

    datm = {k: (dev(v) if isinstance(v, np.ndarray) and k != "slab_nz" else v) for k, v in atm.items()}
    datm["species"] = [{k: dev(v) for k, v in sp.items()} for sp in atm["species"]]
    torch.cuda.synchronize()
    ie_d, flux_d, itop_d = m3d.lte_synthesis_windows(datm, dev(nu), dev(llam), vec, wmu, return_itop=True,
                                                     device=True)
    m3d.synchronize()
    np.testing.assert_array_equal(itop_d.cpu().numpy(), itop_h)
    np.testing.assert_array_equal(flux_d.cpu().numpy(), flux_h)
    # one window of the batch against the oracle
    w = 17
    oie, oflux, oitop = P.lte_synthesis(atm, nu[w], llam[w], vec, wmu)
    np.testing.assert_array_equal(itop_h[..., 32 * w:32 * (w + 1)], oitop)
    np.testing.assert_allclose(flux_h[32 * w:32 * (w + 1)], oflux, rtol=2e-6)


def test_window_batch_rejects(m3d):
    from dispatch_b200 import synth
    atm, nu, llam, vec, wmu = synth.lte_config("c0")
    with pytest.raises(m3d.M3DError, match="nf = 32"):
        m3d.lte_synthesis_windows(atm, nu[:96].reshape(2, 48), llam[:96].reshape(2, 48), vec, wmu)
    bad = llam[:64].reshape(2, 32)[:, ::-1].copy()
    with pytest.raises(m3d.M3DError, match="ascending"):
        m3d.lte_synthesis_windows(atm, nu[:64].reshape(2, 32), bad, vec, wmu)

"""short_char_hermite on the device against the oracle, bit for bit (FP32 with the
FP64 dtau and weights): both directions, oblique rays leaning either way, with and
without the Lambda diagonal and the split rates, on a smooth stratified slab and on
one with rough chi and Snu (every branch of the slope clamps), a maser cell
included."""
import numpy as np
import pytest

from hermite_cases import HERM3D_KEYS, slab_case3d

pytestmark = pytest.mark.gpu


def _case(rough, seed=7):
    work, fld, ds = slab_case3d(seed=seed)
    if rough:
        rng = np.random.default_rng(seed)
        work[0] *= (1 + 0.6 * rng.random(work[0].shape)).astype(np.float32)
        work[1] *= (1 + 0.4 * rng.standard_normal(work[1].shape) ** 2).astype(np.float32)
        work[0, 3, 2, 4, 1] = -0.3 * work[0, 3, 2, 4, 1]          # a maser cell
    return work, fld, ds


@pytest.mark.parametrize("dir", [1, -1])
@pytest.mark.parametrize("psi_on,split", [(True, False), (True, True), (False, False), (False, True)])
@pytest.mark.parametrize("rough", [False, True])
@pytest.mark.parametrize("lean", [1.0, -1.0])
def test_short_char_hermite_bit_exact(m3d, oracle, dir, psi_on, split, rough, lean):
    work, fld, ds = _case(rough)
    nz, ny, nx, nf = work.shape[1] - 2, work.shape[2], work.shape[3], work.shape[4]
    vec = np.array([0.3 * lean, -0.2, 0.0])
    vec[2] = dir * np.sqrt(1 - 0.13)
    zg = 0 if dir > 0 else nz + 1
    work[2, zg] = work[1, zg]
    out = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        w = work.copy()
        bufs = [np.full((nz, ny, nx, nf), -7.0, np.float32) for _ in range(3)]
        slab = mod.make_slab(nf, nx, ny, nz, dir, [ds, ds, ds], vec, get_psi=psi_on, split_rates=split)
        fn = oracle.short_char_hermite if name == "o" else m3d.rt.short_char_hermite
        fn(slab, w, bufs[0] if psi_on else None, bufs[1] if split else None, bufs[2] if split else None,
           *[fld[k] for k in HERM3D_KEYS])
        out[name] = (w, *bufs)
    for a, b in zip(out["g"], out["o"]):
        np.testing.assert_array_equal(a, b)
    assert np.isfinite(out["o"][0]).all()
    if psi_on:
        assert out["o"][1].max() > 0


def test_short_char_hermite_device_tensors_and_checks(m3d):
    """Device tensors in place equal the host call; a ray whose upwind point lies
    beyond one cell and split rates without their buffers are rejected."""
    import torch
    work, fld, ds = _case(False)
    nz, ny, nx, nf = work.shape[1] - 2, work.shape[2], work.shape[3], work.shape[4]
    work[2, 0] = work[1, 0]
    vec = np.array([0.3, 0.2, np.sqrt(1 - 0.13)])
    slab = m3d.make_slab(nf, nx, ny, nz, 1, [ds] * 3, vec, get_psi=True, split_rates=True)
    h = [np.zeros((nz, ny, nx, nf), np.float32) for _ in range(3)]
    w_h = work.copy()
    m3d.rt.short_char_hermite(slab, w_h, *h, *[fld[k] for k in HERM3D_KEYS])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    w_d = dev(work)
    d = [torch.zeros(h[0].shape, dtype=torch.float32, device="cuda") for _ in range(3)]
    m3d.rt.short_char_hermite(slab, w_d, *d, *[dev(fld[k]) for k in HERM3D_KEYS])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(w_d.cpu().numpy(), w_h)
    for a, b in zip(d, h):
        np.testing.assert_array_equal(a.cpu().numpy(), b)
    steep = m3d.make_slab(nf, nx, ny, nz, 1, [ds] * 3, [0.9, 0.0, np.sqrt(1 - 0.81)])
    with pytest.raises(m3d.M3DError, match="cells away"):
        m3d.rt.short_char_hermite(steep, work.copy(), None, None, None, *[fld[k] for k in HERM3D_KEYS])
    with pytest.raises(m3d.M3DError, match="split_rates without"):
        m3d.rt.short_char_hermite(slab, work.copy(), h[0], None, None, *[fld[k] for k in HERM3D_KEYS])

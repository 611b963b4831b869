"""long_char_hermite and long_char_hermite2 on the device against the oracle (bit
for bit, FP32 with hermite2's FP64 dtau and weights): both directions, the ghost's
state given or the zeroed ghost's secant step, with and without the Lambda
diagonal; hermite2 also on slabs of 2 and 3 planes and with both ghost kinds."""
import numpy as np
import pytest

from hermite_cases import slab_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dir", [1, -1])
@pytest.mark.parametrize("ghost", [True, False])
@pytest.mark.parametrize("psi_on", [True, False])
def test_long_char_hermite_bit_exact(m3d, oracle, dir, ghost, psi_on):
    work, fld, ghosts, ds = slab_case(seed=5 + dir)
    nz, ny, nx, nf = work.shape[1] - 2, work.shape[2], work.shape[3], work.shape[4]
    vec = np.array([0.3, -0.2, 0.0])
    vec[2] = dir * np.sqrt(1 - 0.13)
    g = ghosts["bottom" if dir > 0 else "top"] if ghost else None
    out = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        w = work.copy()
        zg = 0 if dir > 0 else nz + 1
        if not ghost:
            w[:, zg] = 0.0                    # the zeroed ghost of set_upstream_boundary's top branch
        else:
            w[2, zg] = w[1, zg]               # the LTE ghost: Inu = Snu
        psi = np.zeros((nz, ny, nx, nf), np.float32)
        slab = mod.make_slab(nf, nx, ny, nz, dir, [ds * 1.5, ds * 1.5, ds], vec, get_psi=psi_on)
        args = [fld[k] for k in ("beta", "pe", "dpe_dz", "dlnt_dz", "temp", "hknu")]
        if name == "o":
            oracle.long_char_hermite(slab, w, psi, *args, ghost=g)
        else:
            m3d.rt.long_char_hermite(slab, w, psi, *args, ghost=g)
        out[name] = (w, psi)
    np.testing.assert_array_equal(out["g"][0], out["o"][0])
    np.testing.assert_array_equal(out["g"][1], out["o"][1])
    assert np.isfinite(out["o"][0]).all()
    if psi_on:
        assert out["o"][1].max() > 0


def test_long_char_hermite_rejects_thin_slab(m3d):
    work, fld, ghosts, ds = slab_case(nz=2)
    slab = m3d.make_slab(work.shape[4], work.shape[3], work.shape[2], 2, 1, [ds] * 3, [0, 0, 1.0])
    with pytest.raises(m3d.M3DError, match="nz >= 3"):
        m3d.rt.long_char_hermite(slab, work, None, *[fld[k] for k in ("beta", "pe", "dpe_dz", "dlnt_dz", "temp",
                                                                       "hknu")])


@pytest.mark.parametrize("dir", [1, -1])
@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("nz", [9, 3, 2])
def test_long_char_hermite2_bit_exact(m3d, oracle, dir, kind, nz):
    work, fld, ghosts, ds = slab_case(seed=11 + dir + nz, nz=nz)
    ny, nx, nf = work.shape[2], work.shape[3], work.shape[4]
    vec = np.array([0.2, 0.1, 0.0])
    vec[2] = dir * np.sqrt(1 - 0.05)
    g = ghosts["bottom" if dir > 0 else "top"] if kind else None
    out = {}
    for name, mod in (("o", oracle), ("g", m3d)):
        w = work.copy()
        zg = 0 if dir > 0 else nz + 1
        if not kind:
            w[:, zg] = 0.0
        else:
            w[2, zg] = w[1, zg]
        psi = np.zeros((nz, ny, nx, nf), np.float32)
        slab = mod.make_slab(nf, nx, ny, nz, dir, [ds * 1.5, ds * 1.5, ds], vec, get_psi=True)
        fn = oracle.long_char_hermite2 if name == "o" else m3d.rt.long_char_hermite2
        fn(slab, w, psi, fld["pe"], fld["dpe_dz"], ghost=g, ghost_kind=kind)
        out[name] = (w, psi)
    np.testing.assert_array_equal(out["g"][0], out["o"][0])
    np.testing.assert_array_equal(out["g"][1], out["o"][1])
    assert np.isfinite(out["o"][0]).all()
    assert out["o"][1].max() > 0


def test_long_char_hermite2_device_buffers_and_checks(m3d, oracle):
    """Device tensors in place equal the host call; a 1-plane slab, a ghost kind
    out of range and a ghost kind without its Pe are rejected."""
    import torch
    work, fld, ghosts, ds = slab_case(seed=4, nz=6)
    nz, ny, nx, nf = 6, work.shape[2], work.shape[3], work.shape[4]
    slab = m3d.make_slab(nf, nx, ny, nz, 1, [ds] * 3, [0.0, 0.0, 1.0], get_psi=True)
    w_h = work.copy()
    w_h[2, 0] = w_h[1, 0]
    w_d = torch.from_numpy(w_h.copy()).cuda()
    psi_h = np.zeros((nz, ny, nx, nf), np.float32)
    psi_d = torch.zeros(psi_h.shape, dtype=torch.float32, device="cuda")
    gb = ghosts["bottom"]
    m3d.rt.long_char_hermite2(slab, w_h, psi_h, fld["pe"], fld["dpe_dz"], ghost=gb)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    m3d.rt.long_char_hermite2(slab, w_d, psi_d, dev(fld["pe"]), dev(fld["dpe_dz"]),
                              ghost={k: dev(v) for k, v in gb.items()})
    torch.cuda.synchronize()
    np.testing.assert_array_equal(w_d.cpu().numpy(), w_h)
    np.testing.assert_array_equal(psi_d.cpu().numpy(), psi_h)
    thin = m3d.make_slab(nf, nx, ny, 1, 1, [ds] * 3, [0.0, 0.0, 1.0])
    with pytest.raises(m3d.M3DError, match="nz >= 2"):
        m3d.rt.long_char_hermite2(thin, work[:, :3].copy(), None, fld["pe"][:1], fld["dpe_dz"][:1])
    import ctypes as C
    lib = m3d.lib()
    for kind, gp in ((3, None), (1, None)):
        rc = lib.m3d_long_char_hermite2(C.byref(slab), m3d.ptr(w_h), None, m3d.ptr(fld["pe"]),
                                        m3d.ptr(fld["dpe_dz"]), gp, gp, C.c_int(kind), C.c_double(1.0),
                                        C.c_uint(0))
        assert rc != 0

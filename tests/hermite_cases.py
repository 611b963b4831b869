"""A stratified LTE slab for the Hermite solver tests: temperature falling and
electron pressure falling exponentially upwards, chi tied to Pe, Snu = Bnu(T), the
d/dz by centred differences, small horizontal fluctuations."""
import numpy as np


def slab_case(seed=3, nf=6, nx=5, ny=4, nz=9, ds=2e6):
    rng = np.random.default_rng(seed)
    z = np.arange(nz + 2, dtype=np.float64)                     # ghost 0 .. nz+1, bottom at 0
    h = z / (nz + 1)                                            # 0 at the bottom ghost, 1 at the top one
    T = (9000.0 - 4000.0 * h)[:, None, None] * (1 + 0.02 * rng.standard_normal((nz + 2, ny, nx)))
    Pe = (300.0 * np.exp(-4.0 * h))[:, None, None] * (1 + 0.05 * rng.standard_normal((nz + 2, ny, nx)))
    hknu = np.linspace(2.4e4, 3.2e4, nf).astype(np.float32)     # h nu / k for 4500-6000 A
    beta = np.exp(-hknu[None, None, None, :] / T[..., None])
    B = beta / (1 - beta)
    chi = (2e-7 * (Pe / 300.0) ** 0.7)[..., None] * (1 + 0.5 * rng.random((nz + 2, ny, nx, nf)))
    work = np.zeros((3, nz + 2, ny, nx, nf), np.float32)
    work[0] = chi
    work[1] = B
    dlnt = np.gradient(np.log(T), axis=0) / ds                  # per cm (code length 1 cm)
    dpe = np.gradient(Pe, axis=0) / ds
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    inner = slice(1, nz + 1)
    fields = {"beta": f32(beta[inner]), "pe": f32(Pe[inner]), "dpe_dz": f32(dpe[inner]),
              "dlnt_dz": f32(dlnt[inner]), "temp": f32(T[inner]), "hknu": hknu}
    ghosts = {}
    for name, zi in (("bottom", 0), ("top", nz + 1)):
        ghosts[name] = {"pe": f32(Pe[zi]), "dpe_dz": f32(dpe[zi]), "dlnt_dz": f32(dlnt[zi]), "temp": f32(T[zi])}
    return work, fields, ghosts, ds

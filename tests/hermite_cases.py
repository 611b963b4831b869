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


def slab_case3d(seed=3, nf=5, nx=8, ny=6, nz=7, ds=2e6, amp=0.03):
    """A stratified LTE slab with smooth periodic horizontal waves, for the 3D
    short-characteristics Hermite solver: the fields of slab_case without the
    per-cell noise, plus the horizontal derivatives by periodic centred
    differences (cells ds apart in x, y and z)."""
    rng = np.random.default_rng(seed)
    z = np.arange(nz + 2, dtype=np.float64)
    h = (z / (nz + 1))[:, None, None]
    X = 2 * np.pi * np.arange(nx)[None, None, :] / nx
    Y = 2 * np.pi * np.arange(ny)[None, :, None] / ny
    ph = rng.uniform(0, 2 * np.pi, 3)
    wave = np.sin(X + ph[0]) * np.cos(Y + ph[1]) + 0.5 * np.sin(X - Y + ph[2])
    T = (9000.0 - 4000.0 * h) * (1 + amp * wave)
    Pe = 300.0 * np.exp(-4.0 * h) * (1 + 2 * amp * wave)
    hknu = np.linspace(2.4e4, 3.2e4, nf).astype(np.float32)
    beta = np.exp(-hknu[None, None, None, :] / T[..., None])
    B = beta / (1 - beta)
    chi = (2e-7 * (Pe / 300.0) ** 0.7)[..., None] * np.linspace(1.0, 1.5, nf)[None, None, None, :]
    work = np.zeros((3, nz + 2, ny, nx, nf), np.float32)
    work[0] = chi
    work[1] = B
    lnT = np.log(T)
    dx = lambda a: (np.roll(a, -1, axis=2) - np.roll(a, 1, axis=2)) / (2 * ds)
    dy = lambda a: (np.roll(a, -1, axis=1) - np.roll(a, 1, axis=1)) / (2 * ds)
    dz = lambda a: np.gradient(a, axis=0) / ds
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    inner = slice(1, nz + 1)
    fields = {"beta": f32(beta[inner]), "pe": f32(Pe[inner]), "temp": f32(T[inner]), "hknu": hknu,
              "dpe_dx": f32(dx(Pe)[inner]), "dpe_dy": f32(dy(Pe)[inner]), "dpe_dz": f32(dz(Pe)[inner]),
              "dlnt_dx": f32(dx(lnT)[inner]), "dlnt_dy": f32(dy(lnT)[inner]), "dlnt_dz": f32(dz(lnT)[inner])}
    return work, fields, ds


HERM3D_KEYS = ("beta", "pe", "dpe_dx", "dpe_dy", "dpe_dz", "dlnt_dx", "dlnt_dy", "dlnt_dz", "temp", "hknu")

"""Seeded cells and sampled opacity tables for the table tests, plus a numpy
restatement of the table's node slopes (pchip_slopes8 / pchip_slopes4 of
interpol_mod.f90:193-284, vectorised) that cross-checks the C oracle's."""
import numpy as np

from dispatch_b200 import synth


def cells(seed=1, nx=12, ny=10, nz=16):
    return synth.optab_cells(seed, nx, ny, nz)


def table(kind="background", seed=2, nnu=300, scat=True, cells_=None):
    c = cells_ or cells()
    return synth.sample_table(seed, c["temp"], c["ne"], nnu=nnu, kind=kind, scat=scat)


def _ends(first_d, last_d, dy0, dx0, dyl, dxl, two):
    return two * dy0 / dx0 - first_d, two * dyl / dxl - last_d


def slopes_lam(lam, val):
    """pchip_slopes8 along the last axis on fp64 nodes, rounded to fp32."""
    y = val.astype(np.float64)
    dx = np.diff(lam)
    dy = np.diff(y, axis=-1)
    if lam.size == 2:
        a = dy[..., 0] / dx[0]
        a = 2.0 * dy[..., 0] / dx[0] - a
        b = 2.0 * dy[..., 0] / dx[0] - a
        return np.stack([a, b], axis=-1).astype(np.float32)
    dym, dyp, dxm, dxp = dy[..., :-1], dy[..., 1:], dx[:-1], dx[1:]
    with np.errstate(divide="ignore", invalid="ignore"):
        d1, d2 = dym / dxm, dyp / dxp
        ok = (dym != 0) & (dyp != 0) & (np.copysign(1.0, d1) == np.copysign(1.0, d2))
        alpha = (1.0 + dxm / (dxp + dxm)) / 3.0
        d = np.where(ok, 1.0 / ((1.0 - alpha) / d1 + alpha / d2), 0.0)
    s0, sn = _ends(d[..., 0], d[..., -1], dy[..., 0], dx[0], dy[..., -1], dx[-1], 2.0)
    return np.concatenate([s0[..., None], d, sn[..., None]], axis=-1).astype(np.float32)


def slopes_axis(c0, dc, val, axis):
    """pchip_slopes4 along a regular PC axis (fp32 nodes and differences, the
    harmonic mean in fp64), the node slopes pchip_mono4 returns at the nodes."""
    v = np.moveaxis(val, axis, -1).astype(np.float32)
    n = v.shape[-1]
    x = (c0 + np.arange(n, dtype=np.float64) * dc).astype(np.float32)
    dx = np.diff(x)
    dy = np.diff(v, axis=-1)
    f32 = np.float32
    if n == 2:
        a = dy[..., 0] / dx[0]
        a = f32(2) * dy[..., 0] / dx[0] - a
        b = f32(2) * dy[..., 0] / dx[0] - a
        return np.moveaxis(np.stack([a, b], axis=-1), -1, axis)
    dym, dyp, dxm, dxp = dy[..., :-1], dy[..., 1:], dx[:-1], dx[1:]
    with np.errstate(divide="ignore", invalid="ignore"):
        d1, d2 = (dym / dxm).astype(np.float64), (dyp / dxp).astype(np.float64)
        ok = (dym != 0) & (dyp != 0) & (np.copysign(1.0, d1) == np.copysign(1.0, d2))
        alpha = ((f32(1) + dxm / (dxp + dxm)) / f32(3)).astype(np.float64)
        d = np.where(ok, 1.0 / ((1.0 - alpha) / d1 + alpha / d2), 0.0).astype(np.float32)
    s0, sn = _ends(d[..., 0], d[..., -1], dy[..., 0], dx[0], dy[..., -1], dx[-1], f32(2))
    out = np.concatenate([s0[..., None], d, sn[..., None]], axis=-1).astype(np.float32)
    return np.moveaxis(out, -1, axis)


def node_cells(tab, picks):
    """(T, ne) exactly at table nodes (it, je) given as pairs, flat."""
    Tn, Nn = synth.table_nodes(tab["pca"], tab["val"].shape[1], tab["val"].shape[0])
    it = np.array([p[0] for p in picks])
    je = np.array([p[1] for p in picks])
    return Tn[je, it], Nn[je, it]

"""The LTE output pass composed from the oracle's routines, in the reference's
order (rt_patch_t%execute do_final branch, rt_patch_mod.f90:1014-1030, per slab
of rt_column_t%execute, rt_column_mod.f90:252-310).

TEST INFRASTRUCTURE ONLY (checker of m3d_lte_synthesis; CPU baseline of bench.py).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

H_K = 6.626176e-27 / 1.380662e-16


def transfer_units(atm, nu, llam, vec, tol=1e-4, fp64=False):
    """(chi, S) of every cell for direction vec: (ncell, nf), f32 or f64.  fp64: the
    plain FP64 path, line opacity and profile included (oracle.opacity_f64)."""
    if fp64:
        return _transfer_units_f64(atm, nu, llam, vec, tol)
    vx = atm["vx"].astype(np.float64)
    vy = atm["vy"].astype(np.float64)
    vz = atm["vz"].astype(np.float64)
    vproj = ((vec[0] * vx + vec[1] * vy) + vec[2] * vz).astype(np.float32)
    beta, Bnu = O.lte_background(nu, atm["temp"])
    xhat, ehat = O.lte_work(atm["chi_c"], beta, Bnu)
    lr = O.logref(xhat, tol)
    ncell = atm["temp"].size
    chil = np.zeros((ncell, nu.size), np.float32)
    etal = np.zeros_like(chil)
    for sp in atm["species"]:
        cells = {"vproj": vproj, "inv_df": sp["inv_df"], "vbar2": sp["vbar2"], "lnbase": sp["lnbase"],
                 "e_kT": atm["e_kT"], "ne": atm["ne"], "tothi": atm["tothi"], "stark_pe": atm["stark_pe"]}
        O.add_opacity_equi(sp, llam, chil, etal, xhat, lr, cells, tol=tol)
    w1 = (xhat + chil).astype(np.float32)
    w2 = (ehat + etal).astype(np.float32)
    O.work_to_transfer_units(w1, w2, beta, atm.get("maser_chi_floor", 1e-4))
    return w1, w2


def _transfer_units_f64(atm, nu, llam, vec, tol):
    vproj = (vec[0] * atm["vx"].astype(np.float64) + vec[1] * atm["vy"].astype(np.float64)) \
        + vec[2] * atm["vz"].astype(np.float64)
    T = atm["temp"].astype(np.float64)[:, None]
    hv = nu[None, :] * (H_K / T)
    b = np.maximum(np.exp(-hv), np.finfo(np.float64).tiny)
    Bn = b / (-np.expm1(-hv))
    cc = atm["chi_c"].astype(np.float64)[:, None]
    eta_c = cc * Bn
    xhat = cc + eta_c
    chil = np.zeros((atm["temp"].size, nu.size), np.float64)
    for sp in atm["species"]:
        cells = {"inv_df": sp["inv_df"], "vbar2": sp["vbar2"], "lnbase": sp["lnbase"], "e_kT": atm["e_kT"],
                 "ne": atm["ne"], "tothi": atm["tothi"], "stark_pe": atm["stark_pe"]}
        O.opacity_f64(sp, llam, chil, xhat, vproj, cells, tol=tol)
    w1 = xhat + chil
    w2 = eta_c / b + chil
    etav = w2 * b
    chi = w1 - etav
    fl = np.maximum(np.float64(np.float32(atm.get("maser_chi_floor", 1e-4))) * np.abs(w1), np.finfo(np.float64).tiny)
    chi = np.where(np.abs(chi) < fl, np.copysign(fl, chi), chi)
    return chi, etav / chi


def column_sweep(atm, chi, S, vec, fp64=False):
    """Slabs bottom to top: PCHIP ghost, rotate_array (3D only), long_char_quadratic,
    exit plane handed on.  chi, S: (ncell, nf).  Returns the emergent plane
    (ny, nx, nf)."""
    nx, ny, nz = atm["nx"], atm["ny"], atm["nz"]
    nf = chi.shape[1]
    dt = np.float64 if fp64 else np.float32
    chi = chi.reshape(nz, ny, nx, nf)
    S = S.reshape(nz, ny, nx, nf)
    ds_code = atm["ds_code"]
    mem = None
    z0 = 0
    three_d = not (nx == 1 and ny == 1)
    for n in atm["slab_nz"]:
        slab = O.make_slab(nf, nx, ny, n, 1, atm["ds_cm"], vec, maser_dtau_max=atm.get("maser_dtau_max", 2.0),
                           maser_Inu_max=atm.get("maser_Inu_max", 1e30))
        work = np.zeros((3, n + 2, ny, nx, nf), dt)
        work[0, 1:n + 1] = chi[z0:z0 + n]
        work[1, 1:n + 1] = S[z0:z0 + n]
        if mem is None:
            O.upstream_boundary(slab, work, O.BND_PCHIP, ds3_code=np.float32(ds_code[2]))
        else:
            O.upstream_boundary(slab, work, O.BND_NONE, mem=mem)
        if three_d:
            bottom = float(np.float32(z0 * ds_code[2]))
            O.rotate_array(slab, work, ds_code, atm["pivot_z"] - bottom, atm.get("ray_offset", (0.0, 0.0)))
        O.formal_solve(O.QUADRATIC, slab, work)
        mem = np.ascontiguousarray(work[:, n])
        z0 += n
    return mem[2]


def lte_synthesis(atm, nu, llam, vec, wmu, fp64=False, tol=1e-4):
    """Returns (ie (nray, nf), flux (nf,), i_top (nray, ny, nx, nf))."""
    tops = []
    for r in range(wmu.size):
        chi, S = transfer_units(atm, nu, llam, vec[r], tol=tol, fp64=fp64)
        tops.append(column_sweep(atm, chi, S, vec[r], fp64=fp64))
    i_top = np.stack(tops)
    ie, flux = O.save_intensity(nu, i_top.astype(np.float32), wmu)
    return ie, flux, i_top

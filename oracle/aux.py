"""numpy restatement of the auxiliary steps around the solvers.  TEST
INFRASTRUCTURE ONLY: the checker of m3d_update_eta_mask, m3d_lte_populations and
m3d_particle_fields.

  update_eta_mask              SRC/rt_patch_mod.f90:3671-3807 (flags dense, one per point)
  compute_lte_populations      SRC/atom_mod.f90:1041-1140, level partition function
  lte_pop                      SRC/atom_mod.f90:1132-1150
  inverse_doppler_factor,
  compute_vbar2, lnbase        HOP/ion_mod.f90:198-221, HOP/linelist_mod.f90:1023-1042

Arrays are numpy C order with the Fortran index order reversed: work is
(3, nz+2, ny, nx, nf), beta and the flags (nz, ny, nx, nf), the ghost flags (ny, nx, nf).
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32


def eta_fire(chi, one_m_beta, S):
    """min(chi, |chi| - q_eta (chi + (1 - beta) chi S)) <= 0 in float32 (:3722)."""
    chi, one_m_beta, S = F(chi), F(one_m_beta), F(S)
    with np.errstate(all="ignore"):
        t = F(one_m_beta * chi) * S
        v = np.abs(chi) - F(1e-2) * F(chi + t)
        return np.fmin(chi, v) <= F(0)


def update_eta_mask(work, beta, src, gsrc, mask, dir, rx, ry, ghost):
    """In place on src, gsrc, mask (uint8)."""
    nz = beta.shape[0]
    fire = eta_fire(work[0, 1:nz + 1], F(1) - beta, work[1, 1:nz + 1])
    new = fire & (src == 0)
    src |= new.astype(np.uint8)
    z1 = 0 if dir > 0 else nz - 1
    gnew = None
    if ghost:
        zg = 0 if dir > 0 else nz + 1
        gfire = eta_fire(work[0, zg], F(1), work[1, zg])
        gnew = gfire & (gsrc == 0)
        gsrc |= gnew.astype(np.uint8)
    spread = np.zeros_like(new)
    for j in range(-ry, ry + 1):
        for i in range(-rx, rx + 1):
            # a flag at (x, y) reaches (x + i, y + j): roll the source forward
            shifted = np.roll(np.roll(new, j, axis=1), i, axis=2)
            spread |= shifted
            if dir > 0:
                spread[1:] |= shifted[:-1]
            else:
                spread[:-1] |= shifted[1:]
            if gnew is not None:
                spread[z1] |= np.roll(np.roll(gnew, j, axis=0), i, axis=1)
    mask |= spread.astype(np.uint8)


def lte_populations(g, ev, ion, temp, lsaha, dxi, totn):
    """nstar (nlevel, ncell) and the new totn."""
    temp = np.asarray(temp, F)
    ekt = (1.602189e-12 / 1.380662e-16 / temp.astype(np.float64)).astype(F)
    dxi = np.zeros_like(temp) if dxi is None else np.asarray(dxi, F)
    lsaha = np.asarray(lsaha, F)
    nl = len(g)
    ns = np.empty((nl, temp.size))
    for i in range(nl):
        j = int(ion[i])
        low = ((dxi * F(0.5)) * F(j - 1)) * F(j)
        evi = ev[i] - low.astype(np.float64)
        tns = math.log(g[i]) - ekt.astype(np.float64) * evi
        if j > ion[0]:
            tns = tns + (F(j - ion[0]) * lsaha).astype(np.float64)
        ns[i] = np.exp(tns)
    s = np.zeros(temp.size)
    for i in range(nl):
        s = s + ns[i]
    partition = s.astype(F)
    totn = np.asarray(totn, np.float64)
    norm = (totn / partition.astype(np.float64)).astype(F)
    ns = norm.astype(np.float64)[None, :] * ns
    ns[:, totn == 0] = 0.0
    s2 = np.zeros(temp.size)
    for i in range(nl):
        s2 = s2 + ns[i]
    return ns, s2


def particle_fields(awgt, vmic, iso_frac, population_scale, temp, n, part):
    BK, UU, MH, PI, CC = 1.380662e-16, 1.6605655e-24, 1.6726e-24, 3.14159265359, 2.99792458e10
    temp = np.asarray(temp, F)
    cdop, cvb, inv_mh = F(2.0 * BK / UU), F(8.0 * BK / (PI * UU)), F(UU / MH)
    dop = (F(cdop * temp).astype(np.float64) / awgt).astype(F)
    if vmic > 0:
        vm = F(F(vmic) * F(1e5))
        dop = F(dop + F(vm * vm))
    idf = (CC / np.sqrt(dop).astype(np.float64)).astype(F)
    vbar2 = (F(cvb * temp).astype(np.float64) * (float(inv_mh) + 1.0 / awgt)).astype(F)
    lb = np.log(np.maximum(np.asarray(n, np.float64), np.finfo(np.float64).tiny)).astype(F)
    if population_scale > 0:
        lb = F(lb + F(math.log(population_scale)))
    lnbase = (((lb.astype(np.float64) - np.asarray(part, np.float64)) + np.log(idf).astype(np.float64))
              + float(F(math.log(iso_frac)))).astype(F)
    return idf, vbar2, lnbase

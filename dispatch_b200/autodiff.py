"""Differentiable LTE flux spectra: abundance and log gf fits through the library.

The reference fits abundances by finite differences of whole syntheses
(tumult/abundance.py).  Here the flux of a window is a torch.autograd.Function: its
forward is m3d_lte_synthesis (FP32, every ray) and its backward the hand-written
adjoint m3d_lte_synthesis_adjoint, with respect to the pass's own inputs -- temp,
chi_c, e_kT, inv_df, lnbase, gpref.  LteSpectrum forms those inputs in torch from the
physical parameters -- the cell temperatures, the elemental abundances, the lines'
log gf -- as the per-cell fields are formed for add_opacity_equi (HOP/ion_mod.f90:
198-211 for the Doppler factor, HOP/linelist_mod.f90:1000-1047 for lnbase,
HOP/line_types_mod.f90:30-35 for gpref), so torch's autograd carries the gradient the
rest of the way: d flux / d{A_X, log gf, T}.

Tensors live on the GPU; there is no CPU path.
"""
from __future__ import annotations

import math

import numpy as np

from . import order_after_torch
from . import rt
from . import synth


class LteFlux:
    """flux = LteFlux.apply(static, temp, chi_c, e_kT, inv_df, lnbase, gpref).

    static: dict of the window's fixed inputs -- "atm" (geometry and the undifferentiated
    per-cell fields as CUDA tensors), "species" (line lists without gpref, as CUDA
    tensors, plus vbar2), "nu", "llam" (CUDA float64), "vec", "wmu" (numpy).
    inv_df, lnbase: (nspecies, ncell); gpref: every species' lines one after the other."""

    _fn = None

    @classmethod
    def apply(cls, static, temp, chi_c, e_kT, inv_df, lnbase, gpref):
        if cls._fn is None:
            cls._fn = _make_function()
        return cls._fn.apply(static, temp, chi_c, e_kT, inv_df, lnbase, gpref)


def _atm_of(static, temp, chi_c, e_kT, inv_df, lnbase, gpref):
    atm = dict(static["atm"])
    atm["temp"] = temp.detach().contiguous()
    atm["chi_c"] = chi_c.detach().contiguous()
    atm["e_kT"] = e_kT.detach().contiguous()
    species, off = [], 0
    for k, sp in enumerate(static["species"]):
        d = dict(sp)
        n = int(d["llam0"].shape[0])
        d["gpref"] = gpref[off:off + n].detach().contiguous()
        d["inv_df"] = inv_df[k].detach().contiguous()
        d["lnbase"] = lnbase[k].detach().contiguous()
        species.append(d)
        off += n
    atm["species"] = species
    return atm


def _make_function():
    import torch

    class _LteFlux(torch.autograd.Function):
        @staticmethod
        def forward(ctx, static, temp, chi_c, e_kT, inv_df, lnbase, gpref):
            atm = _atm_of(static, temp, chi_c, e_kT, inv_df, lnbase, gpref)
            order_after_torch(atm["temp"])
            _, flux, _ = rt.lte_synthesis(atm, static["nu"], static["llam"], static["vec"], static["wmu"],
                                          device=True)
            ctx.atm, ctx.static = atm, static
            return flux

        @staticmethod
        def backward(ctx, g_flux):
            s = ctx.static
            g = rt.lte_synthesis_adjoint(ctx.atm, s["nu"], s["llam"], s["vec"], s["wmu"],
                                         g_flux.detach().float().contiguous(), device=True)
            return None, g["temp"], g["chi_c"], g["e_kT"], g["inv_df"], g["lnbase"], g["gpref"]

    return _LteFlux


class LteSpectrum:
    """The flux spectrum of a cube, differentiable in the cell temperatures, the
    species' abundances and the lines' log gf.

    atm, raw: a configuration from synth.lte_config_c4 (numpy), raw holding temp, nH,
    the species' masses (awgt), abundances and raw line parameters, and the whole
    frequency grid (llam_all, nu_all).  Windows of 32 frequencies of that grid."""

    NF = 32

    def __init__(self, atm, raw, vec, wmu, vmic_kms=1.0, part=25.0):
        import torch
        dev = "cuda"
        t = lambda a, dt=None: torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=dt)
        self.torch = torch
        fixed = {k: atm[k] for k in ("nx", "ny", "nz", "slab_nz", "ds_cm", "ds_code", "pivot_z", "ray_offset")}
        for k in ("vx", "vy", "vz", "ne", "tothi", "stark_pe"):
            fixed[k] = t(atm[k])
        for k in ("tol", "maser_chi_floor", "maser_dtau_max", "maser_Inu_max"):
            if k in atm:
                fixed[k] = atm[k]
        self.fixed = fixed
        self.chi_c = t(atm["chi_c"])
        self.species = []
        self.gp_const = []
        for sp, rl in zip(atm["species"], raw["lines"]):
            d = {k: t(v) for k, v in sp.items() if k not in ("gpref", "inv_df", "lnbase")}
            self.species.append(d)
            nu0 = synth.HZ_TO_AA / rl["lam"]
            self.gp_const.append(np.log(synth.BIJ_CONST / nu0))
        self.gp_const = t(np.concatenate(self.gp_const), torch.float64)
        self.awgt = [float(a) for a in raw["awgt"]]
        self.ln_nH = t(np.log(raw["nH"]), torch.float64)
        self.vmic2 = float(np.float32((vmic_kms * 1e5) ** 2))
        self.ln_part = float(np.float32(math.log(part)))
        self.llam_all = t(raw["llam_all"], torch.float64)
        self.nu_all = t(raw["nu_all"], torch.float64)
        self.vec = np.ascontiguousarray(vec, np.float64)
        self.wmu = np.ascontiguousarray(wmu, np.float64)
        self.nwin = self.nu_all.shape[0] // self.NF

    def fields(self, temp, abund, loggf):
        """The pass's per-cell and per-line inputs from T (ncell,), A_X (nspecies,) and
        log gf (all lines), as differentiable torch expressions."""
        torch = self.torch
        const = float(np.float32(2.0 * synth.BK / synth.UU))
        idf = torch.stack([synth.CC / torch.sqrt((const * temp) / a + self.vmic2) for a in self.awgt])
        ln_nx = (abund.double()[:, None] - 12.0) * math.log(10.0) + self.ln_nH[None, :]
        lnbase = ln_nx.float() - self.ln_part + torch.log(idf)
        e_kT = float(np.float32(synth.EE / synth.BK)) / temp
        gpref = (loggf.double() * math.log(10.0) + self.gp_const).float()
        return idf, lnbase, e_kT, gpref

    def static(self, window):
        sl = slice(window * self.NF, (window + 1) * self.NF)
        return {"atm": self.fixed, "species": self.species, "nu": self.nu_all[sl].contiguous(),
                "llam": self.llam_all[sl].contiguous(), "vec": self.vec, "wmu": self.wmu}

    def flux(self, temp, abund, loggf, windows):
        """The disk-integrated flux of the given windows, concatenated (float32)."""
        idf, lnbase, e_kT, gpref = self.fields(temp, abund, loggf)
        out = [LteFlux.apply(self.static(w), temp, self.chi_c, e_kT, idf, lnbase, gpref) for w in windows]
        return self.torch.cat(out)

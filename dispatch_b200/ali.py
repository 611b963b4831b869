"""The 3D NLTE ALI iteration of one frequency window, composed from the library's
entry points over device-resident arrays.

One iteration is the ALI branch of rt_patch_t%execute (SRC/rt_patch_mod.f90:1038-1060)
for the two hemisphere twins of a periodic cube held as one patch, then the
atom update of nlte_patch_t%execute (SRC/nlte_patch_mod.f90:590-660):

* per twin: background (lte_background_emission + convert_to_work_units,
  add_bound_free_opacities, :1297-1351); per direction back_to_work, foreground
  (the split start and add_bound_bound_opacities, :1462-1500),
  work_to_transfer_units, set_upstream_boundary, radiative_transfer,
  aniso_integrations (integrate_intensity, bound_bound_rates, :1728-1758); then
  iso_integrations (bound_free_rates, integrate_rates, :1765-1777);
* combine_twin_hemispheres (:1812-1887);
* the update: normalize_profiles (SRC/atom_mod.f90:377-431), update_populations
  with the fused classic_col rates (:439-732), the convergence bookkeeping of
  nlte_patch_t%execute (:711-765) and ng_acceleration (:2469-2548).

Everything per point stays on the GPU between the calls; the host keeps the
scalars of the convergence test and the Ng gate.  Arrays follow the library's
layout: per-point (ncell, nf) frequency fastest with cell = x + nx (y + ny z),
z = 0 the bottom plane; per-level (nlevel, ncell).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import (AUTOTUNE, BND_PCHIP, BND_ZERO, COL_PERPOINT, SHORT_LINEAR, M3DError, check, init, lib, make_slab, nlte,
               order_after_torch, ptr, rt, stateq, synth)


@dataclass
class AliParams:
    """The run parameters the iteration reads (the reference's &rt_params and
    &nlte_params defaults where they exist)."""

    solver: int = SHORT_LINEAR          # rt_iter%solver: short_char ('linear' in 3D)
    bottom: int = BND_PCHIP             # upstream ghost of upward rays at the bottom
    preconditioning: bool = True        # Rybicki-Hummer preconditioning of the rates
    split_rates: bool = True            # rate_formulation = 'largest'
    maser_chi_floor: float = 1e-4
    maser_dtau_max: float = 2.0
    maser_Inu_max: float = 1e30
    se_solver: int = stateq.LINEQ_NO_PIVOT
    max_update: float = 1e2
    sor_w: float = 1.0
    min_pop_frac: float = 1e-30
    convlim: float = 1e-3
    ng_step: int = 0                    # < 0 off, 0 the automatic gate, > 0 fixed schedule
    ng_start: int = 0
    ng: stateq.NgParams = field(default_factory=stateq.NgParams)


class _AtomIteration:
    """The model atom's state on the cells of a sweep, and the update between sweeps
    (nlte_patch_t%execute: normalize_profiles, update_populations, the convergence
    bookkeeping and ng_acceleration)."""

    def _init_atom(self, atom: dict, wins: list, temp, ne, nH, abundance, awgt: float, vmic_kms: float, dev,
                   all_wins: list | None = None):
        import torch

        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
        temp = np.ascontiguousarray(temp, np.float32).ravel()
        ne = np.asarray(ne, np.float64).ravel()
        nH = np.asarray(nH, np.float64).ravel()
        nc = temp.size
        self.atom = atom
        self.ncell = nc
        totn0 = 10.0 ** (np.asarray(abundance, np.float64) - 12.0) * nH
        nstar, totn = synth.lte_populations(atom, temp, ne, totn0)
        self.temp32 = temp
        self.temp, self.ne = f64(temp), f64(ne)
        self.nh1 = f64(synth.hydrogen_ground(nH, ne)) if atom.get("col_hkind") is not None else None
        self.e_kT = f64(synth.EE / synth.BK / temp.astype(np.float64))
        self.nstar, self.totn = f64(nstar), f64(totn)
        self.pop_ratio = torch.ones(nc, dtype=torch.float64, device=dev)
        idf = synth.inverse_doppler_factor(temp, awgt, vmic_kms).astype(np.float32)
        self.idf_host = idf
        self.inv_df = f32(idf)
        vbar2 = synth.compute_vbar2(temp, awgt).astype(np.float32)
        ne32, nh32 = ne.astype(np.float32), nH.astype(np.float32)
        stark = (ne32 * temp ** np.float32(1.0 / 6.0)).astype(np.float32)
        uns = (vbar2.astype(np.float64) ** 0.3 * nH).astype(np.float32)
        self.adamps = [f32(nlte.bb_damping(w, ne32, nh32, vbar2, stark, uns, idf)) for w in wins]
        nl = self.nlevel = int(atom["nlevel"])
        self.nrad = len(atom["ti"])
        self.b = torch.ones((nl, nc), dtype=torch.float64, device=dev)
        self.oldb = torch.zeros((3, nl, nc), dtype=torch.float64, device=dev)
        self.gamma_ij = torch.zeros((self.nrad, nc), dtype=torch.float32, device=dev)
        self.gamma_ji = torch.zeros_like(self.gamma_ij)
        sums = np.zeros(int(atom["nline"]), np.uint8)
        for w in (all_wins if all_wins is not None else wins):
            sums[np.asarray(w["line_ntrans"], np.int64)] = np.asarray(w["sums_over_windows"], np.uint8)
        self.has_wphi = sums
        # profile integrals of the lines whose windows are summed (rows of the others stay 0)
        self.wphi = torch.zeros((max(int(atom["nline"]), 1), nc), dtype=torch.float32, device=dev)
        self.ng = stateq.NgState(params=self.p.ng)
        self.iter = 0
        self.history: list[dict] = []
        self._sweep_maxerr = 0.0
        self._last_maxerr = 0.0
        self._global = 0.0
        self.converged = False
        self.group = None

    def sweep(self) -> None:
        raise NotImplementedError

    def _exchange(self) -> None:
        """With a process group, the rates of every rank's windows summed on all ranks
        (and the first sweep's profile integrals), before the update."""
        if self.group is None:
            return
        from . import shard
        shard.allreduce_rates(self.gamma_ij, self.gamma_ji, self.wphi if self.iter == 0 else None, self.group)

    # ---- nlte_patch_t%execute ----------------------------------------------------------
    def update(self) -> dict:
        """The atom update of iteration self.iter (>= 1): returns its record."""
        p, it = self.p, self.iter
        nlte.normalize_profiles(self.atom, self.nstar, self.wphi, self.gamma_ij, self.gamma_ji, self.has_wphi,
                                first_iter=it == 1)
        stateq.shift_oldb(self.oldb, self.b)
        res, _ = stateq.stateq_update(self.atom, self.b, self.nstar, self.totn, self.e_kT, self.gamma_ij,
                                      self.gamma_ji, temp=self.temp, ne=self.ne, nh1=self.nh1, solver=p.se_solver,
                                      max_update=p.max_update, sor_w=p.sor_w, min_pop_frac=p.min_pop_frac)
        maxerr = float(res["maxerr"])
        self.ng.count_clamped(res["nclamp"], res["ntot"])
        rec = {"iter": it, "maxerr": maxerr, "epos_cell": int(res["epos_cell"]), "epos_level": int(res["epos_level"]),
               "ng": None}
        convmax = 0.1 * max(p.convlim, 0.0)
        atom_converged = abs(maxerr) < convmax
        if p.ng_step >= 0 and not atom_converged:
            ng = stateq.ng_acceleration(self.ng, it, self._global, p.convlim, self.b, self.oldb, self.nstar,
                                        self.totn, extrapolate=abs(maxerr) >= p.convlim, ng_step=p.ng_step,
                                        ng_start=p.ng_start)
            rec["ng"] = ng
        # the sweep bookkeeping of one patch: the Ng gate reads the change of the
        # iteration before the last (self%global = last_maxerr)
        self._last_maxerr = self._sweep_maxerr
        self._sweep_maxerr = maxerr
        self._global = self._last_maxerr
        applied = bool(rec["ng"] and rec["ng"].get("applied"))
        self.converged = atom_converged or (0.0 < abs(maxerr) < p.convlim and not applied)
        self.gamma_ij.zero_()
        self.gamma_ji.zero_()
        self.history.append(rec)
        return rec

    def run(self, maxiter: int) -> list[dict]:
        """Iteration 0 (LTE start, b = 1) and up to maxiter updates, each followed by
        the next iteration's formal solutions unless it converged."""
        if self.iter == 0:
            self.sweep()
            self._exchange()
        while self.iter < maxiter and not self.converged:
            self.iter += 1
            self.update()
            if not self.converged and self.iter < maxiter:
                self.sweep()
                self._exchange()
        return self.history


class AliWindow(_AtomIteration):
    """One frequency window of a model atom on a periodic cube, device resident.

    cube: temp, ne, nH (ncell,), chi_c (ncell,) grey continuum [1/cm], vz (ncell,)
    vertical velocity [c], the shape (nx, ny, nz) and ds (3,) [cm].  atom: a
    model atom (synth.model_atom); win: its transitions on one frequency window
    (synth.atom_window); vec, wts: the directions of both hemispheres with
    mean-intensity weights (synth.lobatto_rays(..., jnu_weights=True)), the
    upward half first.
    """

    def __init__(self, cube: dict, atom: dict, win: dict, vec, wts, params: AliParams | None = None,
                 abundance: float = 7.5, awgt: float = 56.0, vmic_kms: float = 1.0, device: str = "cuda"):
        import torch

        init()
        self.p = params or AliParams()
        self.atom, self.win = atom, win
        self.nx, self.ny, self.nz = (int(v) for v in cube["shape"])
        self.ds = [float(v) for v in cube["ds"]]
        nc = self.nx * self.ny * self.nz
        self.ncell, self.nf = nc, int(win["nf"])
        vec = np.asarray(vec, np.float64)
        wts = np.asarray(wts, np.float64)
        nd = vec.shape[0]
        if nd % 2 or not np.allclose(vec[nd // 2:], -vec[:nd // 2]) or np.any(vec[:nd // 2, 2] <= 0):
            raise M3DError("AliWindow: vec must hold the upward directions, then the same mirrored")
        self.vec, self.wts = vec, wts
        self.wmu = wts.astype(np.float32)
        # wtot = sum(rt_iter%wmu) in real(4), in the order the directions come
        wt = np.float32(0.0)
        for w in self.wmu:
            wt = np.float32(wt + w)
        self.wtot = float(wt)
        dev = torch.device(device)
        self.dev = dev
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)

        wins = self._windows(win)
        self._init_atom(atom, wins, cube["temp"], cube["ne"], cube["nH"], abundance, awgt, vmic_kms, dev)
        nc = self.ncell
        vz = np.ascontiguousarray(cube["vz"], np.float32).ravel()
        self.vproj = [f32(vz * np.float32(v[2])) for v in vec]
        self.chi_c1 = f32(np.asarray(cube["chi_c"], np.float32).ravel())
        # one flat storage per work array, sized for the widest window; each window
        # takes views of its own shape from the front of them
        nfmax = max(int(w["nf"]) for w in wins)
        nwmax = max(max(int(w["nline"]) + int(w["ncont"]), 1) for w in wins)
        self._pt = nc * nfmax

        def flat(n, dt=torch.float32):
            return torch.zeros(n, dtype=dt, device=dev)

        self._st = {k: flat(self._pt) for k in ("psi", "irem", "escape", "xhat", "ehat", "dj", "opac_L", "opac_R",
                                                 "chi_L", "chi_R", "beta", "Bnu", "chi_c")}
        self._st.update({k: flat(self._pt, torch.int32) for k in ("id", "chi_id")})
        self._st["J"], self._st["PsiJ"] = flat(2 * self._pt), flat(2 * self._pt)
        self._st["work"] = flat(3 * (self.nz + 2) * self.ny * self.nx * nfmax)
        self._st["gw_ij"], self._st["gw_ji"] = flat(nwmax * nc), flat(nwmax * nc)
        self._bind(0)

    def _windows(self, win):
        self.wins = [win]
        return self.wins

    def _bind(self, k: int) -> None:
        """The views and tables of window k."""
        from . import make_slab
        win = self.wins[k]
        self.win = win
        self.adamp = self.adamps[k]
        nc, nf = self.ncell, int(win["nf"])
        self.nf = nf
        shp = (nc, nf)
        st = self._st
        v = lambda key: st[key][:nc * nf].view(shp)
        self.psi, self.irem, self.escape = v("psi"), v("irem"), v("escape")
        self.xhat, self.ehat, self.dj = v("xhat"), v("ehat"), v("dj")
        self.split = {"opac_L": v("opac_L"), "opac_R": v("opac_R"), "id": v("id"), "chi_L": v("chi_L"),
                      "chi_R": v("chi_R"), "chi_id": v("chi_id")}
        self.J = st["J"][:2 * nc * nf].view((2,) + shp)
        self.PsiJ = st["PsiJ"][:2 * nc * nf].view((2,) + shp)
        self.work = st["work"][:3 * (self.nz + 2) * self.ny * self.nx * nf].view(3, self.nz + 2, self.ny, self.nx, nf)
        self.w1 = self.work[0, 1:self.nz + 1].view(shp)
        self.w2 = self.work[1, 1:self.nz + 1].view(shp)
        self.inu = self.work[2, 1:self.nz + 1].view(shp)
        nw = max(int(win["nline"]) + int(win["ncont"]), 1)
        self.gw_ij = st["gw_ij"][:nw * nc].view(nw, nc)
        self.gw_ji = st["gw_ji"][:nw * nc].view(nw, nc)
        import torch
        nu = torch.as_tensor(np.ascontiguousarray(win["nu"], np.float64), device=self.dev)
        self.beta, self.Bnu = rt.lte_background(nu, torch.as_tensor(self.temp32, device=self.dev),
                                                out=(v("beta"), v("Bnu")))
        self.chi_c = v("chi_c")
        self.chi_c.copy_(self.chi_c1[:, None].expand(shp))
        self.slabs = [make_slab(nf, self.nx, self.ny, self.nz, 1 if vv[2] > 0 else -1, self.ds, vv, get_psi=True,
                                split_rates=self.p.split_rates, maser_dtau_max=self.p.maser_dtau_max,
                                maser_Inu_max=self.p.maser_Inu_max) for vv in self.vec]

    # ---- rt_patch_t%execute, ALI branch -------------------------------------------------
    def sweep(self) -> None:
        """The formal solutions of every direction of both twins, with J, PsiJ and the
        rates of this iteration accumulated into gamma_ij/ji."""
        p, win = self.p, self.win
        nd = len(self.slabs)
        first = self.iter == 0
        for h in range(2):
            dirs = range(h * nd // 2, (h + 1) * nd // 2)
            # background: the LTE continuum (pure absorption, Jnu = Bnu) in work units,
            # then the bound-free opacities of the current populations
            rt.lte_emission(self.chi_c, self.Bnu, self.beta, jnu_init=1, out=(self.xhat, self.ehat, self.dj))
            nlte.bf_opacity(win, self.b, self.nstar, self.pop_ratio, self.e_kT, self.xhat, self.ehat)
            self.J[h].zero_()
            self.PsiJ[h].zero_()
            self.gw_ij.zero_()
            self.gw_ji.zero_()
            for d in dirs:
                slab, wmu, vp = self.slabs[d], float(self.wmu[d]), self.vproj[d]
                if p.split_rates:
                    # add_bound_bound_opacities and work_to_transfer_units in one pass
                    # from the background to (chi, S)
                    nlte.bb_opacity_units(win, self.b, self.nstar, self.pop_ratio, self.e_kT, self.inv_df, vp,
                                          self.adamp, self.xhat, self.ehat, self.beta, self.w1, self.w2, self.split,
                                          wmu=wmu, wphi=self.wphi if first else None,
                                          maser_chi_floor=p.maser_chi_floor)
                else:
                    self.w1.copy_(self.xhat)
                    self.w2.copy_(self.ehat)
                    nlte.bb_opacity(win, self.b, self.nstar, self.pop_ratio, self.e_kT, self.inv_df, vp, self.adamp,
                                    self.w1, self.w2, lte=False, wmu=wmu, wphi=self.wphi if first else None)
                    rt.work_to_transfer_units(self.w1, self.w2, self.beta, maser_chi_floor=p.maser_chi_floor)
                mode = p.bottom if slab.dir > 0 else BND_ZERO
                rt.upstream_boundary(slab, self.work, mode)
                rt.formal_solve(p.solver, slab, self.work, psi=self.psi,
                                irem=self.irem if p.split_rates else None,
                                escape=self.escape if p.split_rates else None)
                rt.integrate_intensity(wmu, self.inu, self.psi, self.J[h], self.PsiJ[h])
                nlte.bb_rates(win, self.b, self.nstar, self.pop_ratio, self.e_kT, self.inv_df, vp, self.adamp,
                              self.inu, self.beta, self.Bnu, self.gw_ij, self.gw_ji, work1=self.w1, psi=self.psi,
                              irem=self.irem if p.split_rates else None,
                              escape=self.escape if p.split_rates else None,
                              split=self.split if p.split_rates else None, split_rates=p.split_rates,
                              preconditioning=p.preconditioning, per_direction=True, wmu=wmu, wtot=self.wtot)
            if int(win["ncont"]) > 0:
                nlte.bf_rates(win, self.b, self.nstar, self.e_kT, self.J[h], self.PsiJ[h], self.beta, self.gw_ij,
                              self.gw_ji, preconditioning=p.preconditioning)
            nlte.integrate_rates(win, self.gw_ij, self.gw_ji, self.gamma_ij, self.gamma_ji)
        nlte.combine_twins(self.J[0], self.J[1])
        nlte.combine_twins(self.PsiJ[0], self.PsiJ[1])

    def points(self) -> int:
        """Ray-point-frequency visits of one sweep (both twins)."""
        return len(self.slabs) * self.ncell * sum(int(w["nf"]) for w in self.wins)


class AliCube(AliWindow):
    """Every frequency window of a model atom on a periodic cube: the reference's
    n_windows split (ray_patch_mod.f90:97-127), the rates of all windows summed into
    the atom's gamma_ij/ji before each update, so one sweep is a whole ALI iteration's
    formal solutions.  The windows share one set of work arrays, sized for the widest
    (as one rt_patch_t works its windows in turn).  wins: synth.atom_window of each
    window; the rest as AliWindow."""

    def __init__(self, cube: dict, atom: dict, wins: list, vec, wts, params: AliParams | None = None,
                 abundance: float = 7.5, awgt: float = 56.0, vmic_kms: float = 1.0, device: str = "cuda"):
        self._all = list(wins)
        super().__init__(cube, atom, wins[0], vec, wts, params=params, abundance=abundance, awgt=awgt,
                         vmic_kms=vmic_kms, device=device)

    def _windows(self, win):
        self.wins = self._all
        return self.wins

    def sweep(self) -> None:
        for k in range(len(self.wins)):
            self._bind(k)
            AliWindow.sweep(self)


class _ColProblem(C.Structure):
    """m3d_col_problem_t."""

    _fields_ = [("ncol", C.c_int), ("ncell", C.c_int), ("col_off", C.c_void_p), ("dz", C.c_void_p),
                ("nray", C.c_int), ("mu", C.c_void_p), ("wmu", C.c_void_p), ("b", C.c_void_p),
                ("nstar", C.c_void_p), ("pop_ratio", C.c_void_p), ("e_kT", C.c_void_p), ("inv_df", C.c_void_p),
                ("vz", C.c_void_p), ("chi_c", C.c_void_p), ("temp", C.c_void_p), ("maser_dtau_max", C.c_double),
                ("maser_Inu_max", C.c_double), ("maser_chi_floor", C.c_double), ("preconditioning", C.c_int),
                ("bottom", C.c_int), ("nline_atom", C.c_int), ("nrad_atom", C.c_int)]


class AliColumns(_AtomIteration):
    """The batched 1.5D ALI: columns of uneven depth for one model atom over its
    frequency windows, through the library's column plan (m3d_col_plan_*).

    cols: synth.column_set (cells of every column back to back, abundance variants
    packed as further columns); wins: the atom's frequency windows
    (synth.atom_window with transition subsets); mu, wmu: the directions with
    mean-intensity weights, the upward half first (synth.radau_rays(2,
    jnu_weights=True)[...,2] in 1D).  Each sweep is the plan's fixed launch
    sequence, replayed from a CUDA graph when use_graph; the update between sweeps
    is the base class's.  With autotune the plan times the column solver's launch
    shapes once.  With a process group the windows are shared out over its ranks
    (every world-th one, or the indices given as windows) and run() sums the rates
    over the ranks before each update (shard.allreduce_rates).
    """

    def __init__(self, cols: dict, atom: dict, wins: list, mu, wmu, params: AliParams | None = None,
                 abundance: float = 7.5, awgt: float = 56.0, vmic_kms: float = 1.0, use_graph: bool = True,
                 autotune: bool = True, device: str = "cuda", group=None, windows=None, fused: bool = True):
        import torch

        init()
        self.p = params or AliParams()
        dev = torch.device(device)
        self.dev = dev
        all_wins = list(wins)
        if group is not None and windows is None:
            # frequency windows across the ranks of group: this rank's plan holds every
            # world-th window, and run() sums the rates over the ranks (shard.py)
            import torch.distributed as dist

            from . import shard
            windows = shard.windows_for_rank(dist.get_rank(group), dist.get_world_size(group), len(all_wins))
        if windows is not None:
            if not len(windows):
                raise M3DError(f"AliColumns: no window of {len(all_wins)} for this plan")
            self.wins = [all_wins[w] for w in windows]
        else:
            self.wins = all_wins
        self.use_graph = bool(use_graph)
        abund = abundance + np.asarray(cols.get("abund_dex", 0.0), np.float64)
        self._init_atom(atom, self.wins, cols["temp"], cols["ne"], cols["nH"], abund, awgt, vmic_kms, dev,
                        all_wins=all_wins)
        self.group = group
        nc = self.ncell
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
        self.col_off = torch.as_tensor(np.asarray(cols["col_off"], np.int32), device=dev)
        self.dz = torch.as_tensor(np.asarray(cols["dz"], np.float64), device=dev)
        self.ncol = int(self.col_off.numel()) - 1
        self.vz, self.chi_c, self.tempd = f32(cols["vz"]), f32(cols["chi_c"]), f32(cols["temp"])
        self.mu = np.ascontiguousarray(mu, np.float64)
        self.wmu = np.ascontiguousarray(wmu, np.float32)
        self.nf = [int(w["nf"]) for w in self.wins]
        prob = _ColProblem(self.ncol, nc, self.col_off.data_ptr(), self.dz.data_ptr(), len(self.mu),
                           self.mu.ctypes.data, self.wmu.ctypes.data, self.b.data_ptr(), self.nstar.data_ptr(),
                           self.pop_ratio.data_ptr(), self.e_kT.data_ptr(), self.inv_df.data_ptr(),
                           self.vz.data_ptr(), self.chi_c.data_ptr(), self.tempd.data_ptr(), self.p.maser_dtau_max,
                           self.p.maser_Inu_max, self.p.maser_chi_floor, int(self.p.preconditioning),
                           int(self.p.bottom), int(atom["nline"]), self.nrad)
        nw = len(self.wins)
        ws = (nlte.AtomWindow * nw)()
        self._keep = []
        nus, twos = [], []
        for i, w in enumerate(self.wins):
            st, keep = nlte.make_window(w)
            ws[i] = st
            self._keep.append(keep)
            nus.append(np.ascontiguousarray(w["nu"], np.float64))
            twos.append(np.ascontiguousarray(w["twohnu3_c2"], np.float32))
        self._keep += [nus, twos]
        pv = lambda arrs: (C.c_void_p * nw)(*[a.ctypes.data for a in arrs])
        ad = (C.c_void_p * nw)(*[a.data_ptr() if a.numel() else None for a in self.adamps])
        order_after_torch(self.b)
        self._plan = C.c_void_p()
        check(lib().m3d_col_plan_create(C.byref(prob), C.c_int(nw), ws, pv(nus), pv(twos), ad,
                                        C.c_uint((AUTOTUNE if autotune else 0) | (0 if fused else COL_PERPOINT)),
                                        C.byref(self._plan)),
              "m3d_col_plan_create")
        nfo, blk = C.c_int(), C.c_int()
        check(lib().m3d_col_plan_fields(self._plan, None, None, C.byref(nfo), C.byref(blk)), "m3d_col_plan_fields")
        self.solver_block = blk.value
        sh = [C.c_int() for _ in range(4)]
        check(lib().m3d_col_plan_shape(self._plan, *[C.byref(v) for v in sh]), "m3d_col_plan_shape")
        # the windows the fused kernel sweeps, its threads per column and cells per
        # chunk, the per-point column solver's block size
        self.shape = dict(zip(("fused_windows", "fused_block", "zchunk", "solver_block"), [v.value for v in sh]))

    def sweep(self) -> None:
        """The formal solutions and rate sums of every window and direction."""
        order_after_torch(self.b)
        check(lib().m3d_col_plan_sweep(self._plan, C.c_int(int(self.iter == 0)), ptr(self.gamma_ij),
                                       ptr(self.gamma_ji), ptr(self.wphi), C.c_int(int(self.use_graph))),
              "m3d_col_plan_sweep")

    def fields(self):
        """(J, PsiJ) of the last window, 2 x (ncell, nf) torch tensors (the twins combined)."""
        import torch

        n = (2, self.ncell, self.nf[-1])
        J = torch.empty(n, dtype=torch.float32, device=self.dev)
        P = torch.empty_like(J)
        order_after_torch(J)
        check(lib().m3d_col_plan_fields(self._plan, ptr(J), ptr(P), None, None), "m3d_col_plan_fields")
        return J, P

    def points(self) -> int:
        """Ray-point-frequency visits of one sweep over every window."""
        return len(self.mu) * self.ncell * sum(self.nf)

    def close(self) -> None:
        if getattr(self, "_plan", None) is not None and self._plan.value:
            lib().m3d_col_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def column_problem(kind: str = "small", seed: int = 3, ncol: int = 6, depth=(8, 16), nz: int = 16, nxy: int = 4,
                   nbound: int = 5, nline: int = 6, nper: int = 25, nwin: int = 2, variants=(0.0,),
                   ntheta: int = 2):
    """(cols, atom, wins, mu, wmu) of the batched 1.5D configuration: columns of
    uneven depth from a seeded cube, a model atom split into nwin frequency windows
    (its transitions dealt round-robin), and Radau directions with mean-intensity
    weights.  kind 'c3': 4096 columns of 60-256 cells from a 64 x 64 x 256 cube,
    the 20-level atom (nline 60) in windows of about 10 transitions, abundance
    variants 0 and +-0.2 dex."""
    if kind == "c3":
        ncol, depth, nz, nxy = 4096, (60, 256), 256, 64
        variants = (0.0, 0.2, -0.2)
        nbound, nline, nwin = 20, 60, 8
    cols = synth.column_set(seed, ncol=ncol, depth=depth, nz=nz, nxy=nxy, variants=variants)
    atom = synth.model_atom(seed, nbound=nbound, nline=nline)
    nrad = len(atom["ti"])
    wins = [synth.atom_window(atom, nper=nper, seed=seed, transitions=list(range(k, nrad, nwin)))
            for k in range(nwin)]
    vec, wts = synth.radau_rays(ntheta, 1, jnu_weights=True)
    return cols, atom, wins, vec[:, 2].copy(), wts


# The 3D NLTE configuration's atom draws its lines between levels at least this far
# apart [eV]: with the level energies drawn uniformly, pairs a few meV apart give
# mm-wave lines whose masers drive the iteration to the update limiter.
C2_MIN_LINE_EV = 0.5


def cube_problem(kind: str = "small", seed: int = 2, nx: int = 8, ny: int = 8, nz: int = 12, nbound: int = 6,
                 nline: int = 8, nper: int = 25, transitions=None, ntheta: int = 2, nphi: int = 4,
                 sums=None, min_line_ev: float | None = None) -> tuple[dict, dict, dict, np.ndarray, np.ndarray]:
    """(cube, atom, win, vec, wts) of a seeded NLTE window: the grey cube with its
    temperature and velocity fields, a model atom with nbound bound levels and
    nline lines, its transitions on one window, and Lobatto directions with
    mean-intensity weights.  kind 'c2': the 120^3 cube and the 20-level atom, its
    lines between levels at least 0.5 eV apart (min_line_ev; default 0 otherwise).
    The horizontal cell size is the vertical one times the largest |tan theta| of
    the directions (rounded up to a half), so that every upwind point of the
    short characteristics lies within one cell (the stencil of set_stencil)."""
    if kind == "c2":
        nx = ny = nz = 120
        nbound, nline = 20, 60
        ntheta, nphi = 4, 4
        if min_line_ev is None:
            min_line_ev = C2_MIN_LINE_EV
    vec, wts = synth.lobatto_rays(ntheta, nphi, jnu_weights=True)
    tan_max = float(np.max(np.hypot(vec[:, 0], vec[:, 1]) / np.abs(vec[:, 2])))
    aspect = max(2.0, float(np.ceil(2.0 * tan_max * (1.0 + 1e-6)) / 2.0))
    c = synth.cube_atmosphere(seed, nx, ny, nz, aspect=aspect)
    cube = {"temp": c["temp"].ravel(), "ne": c["ne"].ravel(), "nH": c["nH"].ravel(), "chi_c": c["chi_c"].ravel(),
            "vz": c["vz"].ravel(), "shape": (nx, ny, nz), "ds": c["ds_cm"]}
    atom = synth.model_atom(seed, nbound=nbound, nline=nline, min_line_ev=min_line_ev or 0.0)
    win = synth.atom_window(atom, nper=nper, seed=seed, transitions=transitions, sums=sums)
    return cube, atom, win, vec, wts


__all__ = ["AliParams", "AliWindow", "AliCube", "AliColumns", "cube_problem", "column_problem"]

"""CPU restatement of the 3D NLTE ALI iteration of one frequency window.

TEST INFRASTRUCTURE ONLY: the checker of dispatch_b200.ali.  It composes the
oracle's own kernels (oracle.oracle, oracle.nlte, oracle.stateq) on numpy
arrays in the order the reference runs them:

* rt_patch_t%execute, ALI branch (SRC/rt_patch_mod.f90:1038-1060), for the two
  hemisphere twins of one patch: background (:1297-1351), per direction
  back_to_work (:3542-3560), foreground's split start (:1470-1484) and
  add_bound_bound_opacities, work_to_transfer_units, set_upstream_boundary,
  radiative_transfer, integrate_intensity (:3399-3431) and bound_bound_rates;
  then bound_free_rates and integrate_rates (:3193-3259, :3437-3465);
  combine_twin_hemispheres (:1812-1887);
* nlte_patch_t%execute (SRC/nlte_patch_mod.f90:590-660, :711-765):
  normalize_profiles with the oldb shift (SRC/atom_mod.f90:377-431),
  update_populations with classic_col rates, and ng_acceleration
  (:2469-2548).  The Ng gate's host state machine (ng_mod.f90:88-229) is the
  one the library's front end carries; its kernels here are the oracle's.

Inputs are the ones dispatch_b200.ali.AliWindow takes.
"""
from __future__ import annotations

import numpy as np

from . import nlte as onlte
from . import oracle as orc
from . import stateq as ostq


def _sweep_twins(S: dict) -> None:
    win, nc, nf = S["win"], S["ncell"], S["nf"]
    nz = S["nz"]
    first = S["iter"] == 0
    nd = len(S["slabs"])
    work = S["work"]
    w1 = work[0, 1:nz + 1].reshape(nc, nf)
    w2 = work[1, 1:nz + 1].reshape(nc, nf)
    inu = work[2, 1:nz + 1].reshape(nc, nf)
    for h in range(2):
        # background: LTE continuum emission, Jnu = Bnu, sigma = 0
        xhat, ehat, _, _ = onlte.lte_emission(S["chi_c"], np.zeros_like(S["Bnu"]), S["Bnu"], S["beta"], jmode=1)
        onlte.bf_opacity(win, S["b"], S["nstar"], S["pop_ratio"], S["e_kT"], xhat, ehat)
        J, PsiJ = S["J"][h], S["PsiJ"][h]
        J[:] = 0
        PsiJ[:] = 0
        gw_ij = np.zeros_like(S["gw_ij"])
        gw_ji = np.zeros_like(S["gw_ji"])
        for d in range(h * nd // 2, (h + 1) * nd // 2):
            slab, wmu, vp = S["slabs"][d], float(S["wmu"][d]), S["vproj"][d]
            w1[:] = xhat
            w2[:] = ehat
            split = S["split"]
            onlte.bb_opacity(win, S["b"], S["nstar"], S["pop_ratio"], S["e_kT"], S["inv_df"], vp, S["adamp"], w1, w2,
                             lte=False, wmu=wmu, split=split, wphi=S["wphi"] if first else None)
            onlte.transfer_units_split(w1, w2, S["beta"], split, maser_chi_floor=1e-4)
            mode = orc.BND_PCHIP if slab.dir > 0 else orc.BND_ZERO
            orc.upstream_boundary(slab, work, mode, ds3_code=1.0)
            orc.formal_solve(orc.SHORT_LINEAR, slab, work, psi=S["psi"], irem=S["irem"], escape=S["escape"])
            orc.integrate_intensity(wmu, inu, S["psi"], J, PsiJ)
            onlte.bb_rates(win, S["b"], S["nstar"], S["pop_ratio"], S["e_kT"], S["inv_df"], vp, S["adamp"], inu,
                           S["beta"], S["Bnu"], gw_ij, gw_ji, work1=w1, psi=S["psi"], irem=S["irem"],
                           escape=S["escape"], split=split, split_rates=True, preconditioning=True,
                           per_direction=True, wmu=wmu, wtot=S["wtot"])
        if int(win["ncont"]) > 0:
            onlte.bf_rates(win, S["b"], S["nstar"], S["e_kT"], J, PsiJ, S["beta"], gw_ij, gw_ji,
                           preconditioning=True)
        # integrate_rates: the window's rates into the atom's, by transition index
        nl = int(win["nline"])
        for i, k in enumerate(np.asarray(win["line_ntrans"], np.int64)):
            S["gamma_ij"][k] = S["gamma_ij"][k] + gw_ij[i]
            S["gamma_ji"][k] = S["gamma_ji"][k] + gw_ji[i]
        for i, k in enumerate(np.asarray(win["cont_ntrans"], np.int64)):
            S["gamma_ij"][k] = S["gamma_ij"][k] + gw_ij[nl + i]
            S["gamma_ji"][k] = S["gamma_ji"][k] + gw_ji[nl + i]
    for a in (S["J"], S["PsiJ"]):
        m = ((a[0] + a[1]) * np.float32(0.5)).astype(np.float32)
        a[0] = m
        a[1] = m


def _update(S: dict, ng_state, convlim: float, ng_step: int) -> dict:
    it = S["iter"]
    onlte.normalize_profiles(S["atom"], S["nstar"], S["wphi"], S["gamma_ij"], S["gamma_ji"], S["has_wphi"],
                             first_iter=it == 1)
    oldb = S["oldb"]
    oldb[0] = oldb[1]
    oldb[1] = oldb[2]
    oldb[2] = S["b"]
    res, _, rc = ostq.stateq_update(S["atom"], S["b"], S["nstar"], S["totn"], S["e_kT"], S["gamma_ij"],
                                    S["gamma_ji"], temp=S["temp"], cup=S["cup"], solver=0)
    if rc != 0:
        raise RuntimeError(f"oracle update_populations status {rc}")
    maxerr = float(res["maxerr"])
    ng_state.count_clamped(res["nclamp"], res["ntot"])
    rec = {"iter": it, "maxerr": maxerr, "ng": None}
    atom_converged = abs(maxerr) < 0.1 * max(convlim, 0.0)
    if ng_step >= 0 and not atom_converged:
        out = {"applied": False, "reason": "decided"}
        ng_state.promote(it)
        if it > ng_state.iter_decided:
            ng_state.iter_decided = it
            if ng_step > 0:
                fire = (it % ng_step) == 1 and ng_state.s_done > 0.0
            else:
                fire, out["reason"] = ng_state.should_fire(it, S["global"], convlim)
            if fire:
                ng_state.coefficients()
                ng_state.iter_fired = it
        if ng_state.coeff_valid and ng_state.iter_fired == it and abs(maxerr) >= convlim:
            out.update(ostq.ng_extrapolate(S["b"], oldb, S["nstar"], S["totn"], ng_state.a, ng_state.b,
                                           ng_state.params.max_change))
        if it >= 3 and ng_state.iter_fired != it:
            ng_state.add_gram(ostq.ng_accumulate(S["b"], oldb))
        rec["ng"] = out
    S["last"] = S["sweep"]
    S["sweep"] = maxerr
    S["global"] = S["last"]
    applied = bool(rec["ng"] and rec["ng"].get("applied"))
    S["converged"] = atom_converged or (0.0 < abs(maxerr) < convlim and not applied)
    S["gamma_ij"][:] = 0
    S["gamma_ji"][:] = 0
    return rec


def setup(cube: dict, atom: dict, win: dict, vec, wts, abundance: float = 7.5, awgt: float = 56.0,
          vmic_kms: float = 1.0) -> dict:
    """The state of iteration 0: LTE populations, b = 1, the window's fixed fields."""
    from dispatch_b200 import synth

    nx, ny, nz = (int(v) for v in cube["shape"])
    nc, nf = nx * ny * nz, int(win["nf"])
    temp = np.ascontiguousarray(cube["temp"], np.float32).ravel()
    ne = np.asarray(cube["ne"], np.float64).ravel()
    nH = np.asarray(cube["nH"], np.float64).ravel()
    nstar, totn = synth.lte_populations(atom, temp, ne, 10.0 ** (abundance - 12.0) * nH)
    e_kT = synth.EE / synth.BK / temp.astype(np.float64)
    idf = synth.inverse_doppler_factor(temp, awgt, vmic_kms).astype(np.float32)
    vbar2 = synth.compute_vbar2(temp, awgt).astype(np.float32)
    ne32, nh32 = ne.astype(np.float32), nH.astype(np.float32)
    stark = (ne32 * temp ** np.float32(1.0 / 6.0)).astype(np.float32)
    uns = (vbar2.astype(np.float64) ** 0.3 * nH).astype(np.float32)
    vec = np.asarray(vec, np.float64)
    wmu = np.asarray(wts, np.float64).astype(np.float32)
    wt = np.float32(0.0)
    for w in wmu:
        wt = np.float32(wt + w)
    beta, Bnu = orc.lte_background(win["nu"], temp)
    vz = np.ascontiguousarray(cube["vz"], np.float32).ravel()
    sums = np.zeros(int(atom["nline"]), np.uint8)
    sums[np.asarray(win["line_ntrans"], np.int64)] = np.asarray(win["sums_over_windows"], np.uint8)
    nw = int(win["nline"]) + int(win["ncont"])
    z = lambda dt=np.float32: np.zeros((nc, nf), dt)
    S = {"win": win, "atom": atom, "ncell": nc, "nf": nf, "nz": nz, "iter": 0,
         "temp": temp.astype(np.float64), "e_kT": e_kT, "nstar": nstar, "totn": totn,
         "pop_ratio": np.ones(nc), "inv_df": idf,
         "adamp": onlte.bb_damping(win, ne32, nh32, vbar2, stark, uns, idf),
         "cup": ostq.collision_rates(atom, temp.astype(np.float64), ne, e_kT),
         "vproj": [vz * np.float32(v[2]) for v in vec], "wmu": wmu, "wtot": float(wt),
         "beta": beta, "Bnu": Bnu,
         "chi_c": np.ascontiguousarray(np.broadcast_to(np.asarray(cube["chi_c"], np.float32).ravel()[:, None],
                                                       (nc, nf))),
         "b": np.ones((int(atom["nlevel"]), nc)), "oldb": np.zeros((3, int(atom["nlevel"]), nc)),
         "gamma_ij": np.zeros((len(atom["ti"]), nc), np.float32), "gamma_ji": np.zeros((len(atom["ti"]), nc),
                                                                                       np.float32),
         "gw_ij": np.zeros((max(nw, 1), nc), np.float32), "gw_ji": np.zeros((max(nw, 1), nc), np.float32),
         "has_wphi": sums, "wphi": np.zeros((max(int(atom["nline"]), 1), nc), np.float32),
         "work": np.zeros((3, nz + 2, ny, nx, nf), np.float32), "psi": z(), "irem": z(), "escape": z(),
         "split": {"opac_L": z(), "opac_R": z(), "id": z(np.int32), "chi_L": z(), "chi_R": z(),
                   "chi_id": z(np.int32)},
         "J": np.zeros((2, nc, nf), np.float32), "PsiJ": np.zeros((2, nc, nf), np.float32),
         "slabs": [orc.make_slab(nf, nx, ny, nz, 1 if v[2] > 0 else -1, cube["ds"], v, get_psi=True,
                                 split_rates=True) for v in vec],
         "sweep": 0.0, "last": 0.0, "global": 0.0, "converged": False}
    return S


def sweep(S: dict) -> None:
    """The formal solutions and rate sums of iteration S['iter']."""
    _sweep_twins(S)


def update(S: dict, ng_state, convlim: float = 1e-3, ng_step: int = 0) -> dict:
    """The atom update of iteration S['iter'] (>= 1)."""
    return _update(S, ng_state, convlim, ng_step)


def run(cube: dict, atom: dict, win: dict, vec, wts, maxiter: int, convlim: float = 1e-3, ng_step: int = 0,
        **kw):
    """Iteration 0 and up to maxiter updates; returns (history, state)."""
    from dispatch_b200.stateq import NgState

    S = setup(cube, atom, win, vec, wts, **kw)
    ng_state = NgState()
    hist = []
    _sweep_twins(S)
    while S["iter"] < maxiter and not S["converged"]:
        S["iter"] += 1
        hist.append(_update(S, ng_state, convlim, ng_step))
        if not S["converged"] and S["iter"] < maxiter:
            _sweep_twins(S)
    return hist, S


# ---- every window of the atom: the n_windows split of one patch -------------------------
def setup_windows(cube: dict, atom: dict, wins: list, vec, wts, **kw) -> list:
    """One state per window (ray_patch_mod.f90:97-127), sharing the atom's arrays: the
    populations, the rates (every window's summed into the same gamma_ij/ji), the
    profile integrals and the iteration bookkeeping of the first."""
    Ss = [setup(cube, atom, w, vec, wts, **kw) for w in wins]
    sums = np.zeros(int(atom["nline"]), np.uint8)
    for w in wins:
        sums[np.asarray(w["line_ntrans"], np.int64)] = np.asarray(w["sums_over_windows"], np.uint8)
    S0 = Ss[0]
    S0["has_wphi"] = sums
    for S in Ss[1:]:
        for k in ("b", "oldb", "gamma_ij", "gamma_ji", "wphi", "has_wphi", "nstar", "totn"):
            S[k] = S0[k]
    return Ss


def run_windows(cube: dict, atom: dict, wins: list, vec, wts, maxiter: int, convlim: float = 1e-3,
                ng_step: int = 0, **kw):
    """Iteration 0 and up to maxiter updates over every window; returns (history, state
    of the first window, which holds the shared arrays)."""
    from dispatch_b200.stateq import NgState

    Ss = setup_windows(cube, atom, wins, vec, wts, **kw)
    S0 = Ss[0]
    ng_state = NgState()
    hist = []

    def sweep_all():
        for S in Ss:
            S["iter"] = S0["iter"]
            _sweep_twins(S)

    sweep_all()
    while S0["iter"] < maxiter and not S0["converged"]:
        S0["iter"] += 1
        hist.append(_update(S0, ng_state, convlim, ng_step))
        if not S0["converged"] and S0["iter"] < maxiter:
            sweep_all()
    return hist, S0


# ---- the batched 1.5D iteration: columns of uneven depth ---------------------------------
def _solve_columns(S: dict, Wd: dict, mu: float) -> None:
    """long_char_linear along every column with its upstream ghost (set_upstream_boundary:
    PCHIP at the bottom for upward rays, zero at the top), one 1-column slab each."""
    nf = Wd["nf"]
    off, dz = S["col_off"], S["dz"]
    d = 1 if mu > 0 else -1
    for c in range(len(off) - 1):
        k0, k1 = int(off[c]), int(off[c + 1])
        nz = k1 - k0
        work = np.zeros((3, nz + 2, 1, 1, nf), np.float32)
        work[0, 1:nz + 1, 0, 0] = Wd["w1"][k0:k1]
        work[1, 1:nz + 1, 0, 0] = Wd["w2"][k0:k1]
        slab = orc.make_slab(nf, 1, 1, nz, d, [dz[c]] * 3, [0.0, 0.0, mu], get_psi=True, split_rates=True)
        mode = S["bottom"] if d > 0 else orc.BND_ZERO
        orc.upstream_boundary(slab, work, mode, ds3_code=1.0)
        psi = np.zeros((nz, 1, 1, nf), np.float32)
        irem, esc = np.zeros_like(psi), np.zeros_like(psi)
        orc.formal_solve(orc.LINEAR, slab, work, psi=psi, irem=irem, escape=esc)
        Wd["inu"][k0:k1] = work[2, 1:nz + 1, 0, 0]
        Wd["psi"][k0:k1] = psi[:, 0, 0]
        Wd["irem"][k0:k1] = irem[:, 0, 0]
        Wd["escape"][k0:k1] = esc[:, 0, 0]


def _sweep_columns(S: dict) -> None:
    first = S["iter"] == 0
    nd = len(S["mu"])
    for Wd in S["wins"]:
        win = Wd["win"]
        nc, nf = S["ncell"], Wd["nf"]
        beta, Bnu = orc.lte_background(win["nu"], S["temp32"])
        chi = np.ascontiguousarray(np.broadcast_to(S["chi_c"][:, None], (nc, nf)))
        z = lambda dt=np.float32: np.zeros((nc, nf), dt)
        split = {"opac_L": z(), "opac_R": z(), "id": z(np.int32), "chi_L": z(), "chi_R": z(), "chi_id": z(np.int32)}
        Wd.update({"w1": z(), "w2": z(), "inu": z(), "psi": z(), "irem": z(), "escape": z()})
        J = np.zeros((2, nc, nf), np.float32)
        PsiJ = np.zeros((2, nc, nf), np.float32)
        ntr = max(int(win["nline"]) + int(win["ncont"]), 1)
        for h in range(2):
            xhat, ehat, _, _ = onlte.lte_emission(chi, np.zeros_like(Bnu), Bnu, beta, jmode=1)
            onlte.bf_opacity(win, S["b"], S["nstar"], S["pop_ratio"], S["e_kT"], xhat, ehat)
            gw_ij = np.zeros((ntr, nc), np.float32)
            gw_ji = np.zeros((ntr, nc), np.float32)
            for d in range(h * nd // 2, (h + 1) * nd // 2):
                mu, wmu = float(S["mu"][d]), float(S["wmu"][d])
                vp = (S["vz"] * np.float32(mu)).astype(np.float32)
                Wd["w1"][:] = xhat
                Wd["w2"][:] = ehat
                onlte.bb_opacity(win, S["b"], S["nstar"], S["pop_ratio"], S["e_kT"], S["inv_df"], vp, Wd["adamp"],
                                 Wd["w1"], Wd["w2"], lte=False, wmu=wmu, split=split,
                                 wphi=S["wphi"] if first else None)
                onlte.transfer_units_split(Wd["w1"], Wd["w2"], beta, split, maser_chi_floor=1e-4)
                _solve_columns(S, Wd, mu)
                orc.integrate_intensity(wmu, Wd["inu"], Wd["psi"], J[h], PsiJ[h])
                onlte.bb_rates(win, S["b"], S["nstar"], S["pop_ratio"], S["e_kT"], S["inv_df"], vp, Wd["adamp"],
                               Wd["inu"], beta, Bnu, gw_ij, gw_ji, work1=Wd["w1"], psi=Wd["psi"],
                               irem=Wd["irem"], escape=Wd["escape"], split=split, split_rates=True,
                               preconditioning=True, per_direction=True, wmu=wmu, wtot=S["wtot"])
            if int(win["ncont"]) > 0:
                onlte.bf_rates(win, S["b"], S["nstar"], S["e_kT"], J[h], PsiJ[h], beta, gw_ij, gw_ji,
                               preconditioning=True)
            nl = int(win["nline"])
            for i, k in enumerate(np.asarray(win["line_ntrans"], np.int64)):
                S["gamma_ij"][k] = S["gamma_ij"][k] + gw_ij[i]
                S["gamma_ji"][k] = S["gamma_ji"][k] + gw_ji[i]
            for i, k in enumerate(np.asarray(win["cont_ntrans"], np.int64)):
                S["gamma_ij"][k] = S["gamma_ij"][k] + gw_ij[nl + i]
                S["gamma_ji"][k] = S["gamma_ji"][k] + gw_ji[nl + i]
        m = ((J[0] + J[1]) * np.float32(0.5)).astype(np.float32)
        mp = ((PsiJ[0] + PsiJ[1]) * np.float32(0.5)).astype(np.float32)
        S["J"] = np.stack([m, m])
        S["PsiJ"] = np.stack([mp, mp])


def setup_columns(cols: dict, atom: dict, wins: list, mu, wmu, abundance: float = 7.5, awgt: float = 56.0,
                  vmic_kms: float = 1.0, bottom: int = orc.BND_PCHIP) -> dict:
    """The state of iteration 0 of the batched 1.5D problem (dispatch_b200.ali.AliColumns)."""
    from dispatch_b200 import synth

    temp = np.ascontiguousarray(cols["temp"], np.float32)
    ne = np.asarray(cols["ne"], np.float64)
    nH = np.asarray(cols["nH"], np.float64)
    nc = temp.size
    abund = abundance + np.asarray(cols.get("abund_dex", 0.0), np.float64)
    nstar, totn = synth.lte_populations(atom, temp, ne, 10.0 ** (abund - 12.0) * nH)
    e_kT = synth.EE / synth.BK / temp.astype(np.float64)
    idf = synth.inverse_doppler_factor(temp, awgt, vmic_kms).astype(np.float32)
    vbar2 = synth.compute_vbar2(temp, awgt).astype(np.float32)
    ne32, nh32 = ne.astype(np.float32), nH.astype(np.float32)
    stark = (ne32 * temp ** np.float32(1.0 / 6.0)).astype(np.float32)
    uns = (vbar2.astype(np.float64) ** 0.3 * nH).astype(np.float32)
    wmu32 = np.asarray(wmu, np.float32)
    wt = np.float32(0.0)
    for w in wmu32:
        wt = np.float32(wt + w)
    sums = np.zeros(int(atom["nline"]), np.uint8)
    for w in wins:
        sums[np.asarray(w["line_ntrans"], np.int64)] = np.asarray(w["sums_over_windows"], np.uint8)
    return {"atom": atom, "ncell": nc, "iter": 0, "temp32": temp, "temp": temp.astype(np.float64),
            "e_kT": e_kT, "nstar": nstar, "totn": totn, "pop_ratio": np.ones(nc), "inv_df": idf,
            "cup": ostq.collision_rates(atom, temp.astype(np.float64), ne, e_kT),
            "vz": np.ascontiguousarray(cols["vz"], np.float32), "chi_c": np.ascontiguousarray(cols["chi_c"], np.float32),
            "col_off": np.asarray(cols["col_off"]), "dz": np.asarray(cols["dz"], np.float64),
            "mu": np.asarray(mu, np.float64), "wmu": wmu32, "wtot": float(wt), "bottom": bottom,
            "wins": [{"win": w, "nf": int(w["nf"]),
                      "adamp": onlte.bb_damping(w, ne32, nh32, vbar2, stark, uns, idf)} for w in wins],
            "b": np.ones((int(atom["nlevel"]), nc)), "oldb": np.zeros((3, int(atom["nlevel"]), nc)),
            "gamma_ij": np.zeros((len(atom["ti"]), nc), np.float32),
            "gamma_ji": np.zeros((len(atom["ti"]), nc), np.float32),
            "has_wphi": sums, "wphi": np.zeros((max(int(atom["nline"]), 1), nc), np.float32),
            "sweep": 0.0, "last": 0.0, "global": 0.0, "converged": False}


def sweep_columns(S: dict) -> None:
    _sweep_columns(S)


def run_columns(cols, atom, wins, mu, wmu, maxiter: int, convlim: float = 1e-3, ng_step: int = 0, **kw):
    """Iteration 0 and up to maxiter updates of the batched 1.5D problem."""
    from dispatch_b200.stateq import NgState

    S = setup_columns(cols, atom, wins, mu, wmu, **kw)
    ng_state = NgState()
    hist = []
    _sweep_columns(S)
    while S["iter"] < maxiter and not S["converged"]:
        S["iter"] += 1
        hist.append(_update(S, ng_state, convlim, ng_step))
        if not S["converged"] and S["iter"] < maxiter:
            _sweep_columns(S)
    return hist, S

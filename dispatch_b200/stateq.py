"""Statistical equilibrium: the FP64 rate-matrix update of every cell and Ng's
acceleration, over libm3dgpu.so (include/m3dgpu.h, m3d_stateq_update and
friends).

The host side of Ng -- the shared state, the promotion of the Gram matrix,
the automatic trigger and the 2x2 solve -- is small scalar logic and lives
here, following ng_mod.f90:113-229 and atom_type%ng_acceleration
(atom_mod.f90:2469-2548); the inner products over all cells and the
extrapolation itself run on the device.

Atoms are dicts of numpy arrays (dispatch_b200.synth.model_atom builds them):
nlevel, g, ev, ion, ti, tj, nline, Aji, active (or None), col_i, col_j,
col_kind, col_fac, optionally col_hkind with awgt (hydrogen recipes), and the
scalar factors fmin, cbbesc, cbfesc, colscale, upsilon_floor, cut_x,
bf_cut_rate, cbbhsc, cbfhsc.  Level and transition indices are 0-based.
Per-cell arrays are numpy (C order (level, cell), i.e. the reference's
(cell, level) with the cell fastest) or torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import DEVICE_PTRS, SE_WARP, M3DError, check, init, lib, order_after_torch, ptr

LINEQ_NO_PIVOT, LINEQ, LU_PARTIAL = 0, 1, 2
COL_REGEMORTER, COL_SEATON = 1, 2
COLH_DRAWIN, COLH_TAKEDA = 1, 2
# gencol's record kinds (atom_mod.f90:2288-2344), by the atom file's keys
GENCOL_KINDS = {"OHM": 1, "OHMEGA": 1, "CE": 2, "CH": 3, "CHI": 4, "CI": 5, "CH0": 6, "UP": 7, "DN": 8}
ENONFINITE = 5


class Atom(C.Structure):
    """m3d_atom_t."""

    _fields_ = [("nlevel", C.c_int), ("nrad", C.c_int), ("nline", C.c_int), ("ncol", C.c_int),
                ("trans_i", C.c_void_p), ("trans_j", C.c_void_p), ("active", C.c_void_p), ("Aji", C.c_void_p),
                ("g", C.c_void_p), ("ev", C.c_void_p), ("ion", C.c_void_p),
                ("col_i", C.c_void_p), ("col_j", C.c_void_p), ("col_kind", C.c_void_p), ("col_fac", C.c_void_p),
                ("fmin", C.c_double), ("cbbesc", C.c_double), ("cbfesc", C.c_double), ("colscale", C.c_double),
                ("upsilon_floor", C.c_double), ("cut_x", C.c_double), ("bf_cut_rate", C.c_double),
                ("col_hkind", C.c_void_p), ("drawin", C.c_double), ("cbbhsc", C.c_double), ("cbfhsc", C.c_double),
                ("gencol", C.c_void_p)]


class Gencol(C.Structure):
    """m3d_gencol_t."""

    _fields_ = [("nrec", C.c_int), ("ntemp", C.c_int), ("tgrid", C.c_void_p), ("lnc", C.c_void_p),
                ("dlnc", C.c_void_p), ("ll", C.c_void_p), ("ul", C.c_void_p), ("kind", C.c_void_p),
                ("collider", C.c_void_p), ("ch0_hmip", C.c_int), ("pad", C.c_int)]


class ColCells(C.Structure):
    """m3d_col_cells_t."""

    _fields_ = [("temp", C.c_void_p), ("ne", C.c_void_p), ("dxi", C.c_void_p), ("nh1", C.c_void_p),
                ("lsaha", C.c_void_p), ("colliders", C.c_void_p), ("ncollider", C.c_int), ("pad", C.c_int)]


class SeParams(C.Structure):
    """m3d_se_params_t."""

    _fields_ = [("max_update", C.c_double), ("sor_w", C.c_double), ("min_pop_frac", C.c_double),
                ("conv_pop_floor", C.c_double), ("tmax_update", C.c_double), ("cswitch", C.c_double),
                ("solver", C.c_int), ("pad", C.c_int)]


class SeResult(C.Structure):
    """m3d_se_result_t."""

    _fields_ = [("maxerr", C.c_double), ("epos_cell", C.c_longlong), ("epos_level", C.c_int), ("pad", C.c_int),
                ("nclamp", C.c_longlong), ("ntot", C.c_longlong), ("nonfinite_cell", C.c_longlong)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class NonFiniteSolution(M3DError):
    """m3d_stateq_update found a cell whose rate equations have no finite solution."""

    def __init__(self, msg: str, result: dict, lvlerr: np.ndarray):
        super().__init__(msg)
        self.result = result
        self.lvlerr = lvlerr


def make_atom(atom: dict) -> tuple[Atom, list]:
    """The m3d_atom_t of an atom dict, and the arrays it points into."""
    keep = []

    def arr_of(v, dtype):
        if v is None:
            return None
        a = np.ascontiguousarray(v, dtype)
        keep.append(a)
        return C.c_void_p(a.ctypes.data)

    def arr(key, dtype):
        return arr_of(atom.get(key), dtype)

    s = Atom()
    s.nlevel = int(atom["nlevel"])
    s.nrad = int(len(atom["ti"]))
    s.nline = int(atom["nline"])
    s.ncol = int(len(atom["col_i"])) if atom.get("col_i") is not None else 0
    s.trans_i, s.trans_j = arr("ti", np.int32), arr("tj", np.int32)
    s.active = arr("active", np.uint8)
    s.Aji = arr("Aji", np.float64)
    s.g, s.ev = arr("g", np.float64), arr("ev", np.float64)
    s.ion = arr("ion", np.int32)
    s.col_i, s.col_j = arr("col_i", np.int32), arr("col_j", np.int32)
    s.col_kind, s.col_fac = arr("col_kind", np.int32), arr("col_fac", np.float32)
    for k, d in (("fmin", float(np.float32(1e-6))), ("cbbesc", 1.0), ("cbfesc", 1.0), ("colscale", 1.0),
                 ("upsilon_floor", 0.0), ("cut_x", 70.0), ("bf_cut_rate", 1.0)):
        setattr(s, k, float(atom.get(k, d)))
    s.col_hkind = arr("col_hkind", np.int32)
    s.drawin = prepare_drawin(float(atom["awgt"])) if s.col_hkind is not None else 0.0
    s.cbbhsc, s.cbfhsc = float(atom.get("cbbhsc", 1.0)), float(atom.get("cbfhsc", 1.0))
    gc = atom.get("gencol")
    if gc is not None and len(gc["ll"]) > 0:
        g = Gencol()
        lnc = np.ascontiguousarray(gc["lnc"], np.float64)
        keep.append(lnc)
        g.nrec, g.ntemp = lnc.shape
        g.lnc = C.c_void_p(lnc.ctypes.data)
        g.tgrid = arr_of(gc["tgrid"], np.float64)
        g.dlnc = arr_of(gc.get("dlnc"), np.float64)
        g.ll, g.ul, g.kind = arr_of(gc["ll"], np.int32), arr_of(gc["ul"], np.int32), arr_of(gc["kind"], np.int32)
        g.collider = arr_of(gc.get("collider"), np.int32)
        g.ch0_hmip = int(bool(gc.get("ch0_hmip", False)))
        keep.append(g)
        s.gencol = C.c_void_p(C.addressof(g))
    return s, keep


# constants of prepare_Drawin (HOP/const_mod.f90:14-47, atom_mod.f90:220-222); ame is
# a default-real literal there, so its single-precision value enters the double
# arithmetic
_PI, _BK, _MH, _RBOHR = 3.14159265359, 1.380662e-16, 1.6726e-24, 5.29177349e-9
_AME = float(np.float32(5.485799e-4))
_AMH = 1.0
_MU_E = _AME / (_AME + _AMH)


def prepare_drawin(awgt: float) -> float:
    """prepare_Drawin (atom_mod.f90:1741-1750): the prefactor of Drawin's hydrogen
    rate, 16 pi a0^2 sqrt(2k / (pi m_H A mu_H)) mu_e / mu_H with mu_H = 1 / (A + 1),
    for an atom of weight awgt [amu]."""
    c = (16 * _PI) * (_RBOHR * _RBOHR)
    mu_h = _AMH / (awgt + _AMH)
    drmu = _PI * _MH * awgt * mu_h
    return c * math.sqrt(2.0 * _BK / drmu) * _MU_E / mu_h


def classic_pairs(ion, cont_up, cdata, ecol=None, hcol=None, e_excitation: str = "regemorter",
                  e_ionisation: str = "seaton", h_excitation: str = "", h_ionisation: str = "",
                  h_forbidden: str = "") -> dict:
    """The level pairs classic_col fills and the recipe of each (atom_mod.f90:1790-1876).

    ion (nlevel): ion stage of each level; cont_up (nlevel): the upper level of
    each level's continuum (-1 without one); cdata (nlevel, nlevel): the pair's
    f value (line) or alpha0 (continuum), 0 for none, read at [i, j]; ecol /
    hcol (nlevel, nlevel) bool or None: the pair has electron / hydrogen data in
    the atom file.  A pair i < j enters when ion(j) >= ion(i), a continuum only
    towards cont_up(i), and one of its recipes is unset by the file.  Returns
    col_i, col_j, col_kind, col_hkind (None when no hydrogen recipe is
    selected) and col_fac.
    """
    ion = np.asarray(ion)
    n = ion.size
    cdata = np.asarray(cdata, np.float32)
    ci, cj, ck, chk, cf = [], [], [], [], []
    for i in range(n):
        for j in range(i + 1, n):
            if ion[j] < ion[i]:
                continue
            cont = bool(ion[j] > ion[i])
            if cont and j != cont_up[i]:
                continue
            has_e = bool(ecol[i, j]) if ecol is not None else False
            has_h = bool(hcol[i, j]) if hcol is not None else False
            if has_e and has_h:
                continue
            fac = float(cdata[i, j])
            kind = 0
            if not has_e:
                if cont and e_ionisation == "seaton":
                    kind = COL_SEATON
                elif not cont and e_excitation == "regemorter":
                    kind = COL_REGEMORTER
            hkind = 0
            if not has_h:
                if not cont and fac == 0 and h_forbidden == "takeda":
                    hkind = COLH_TAKEDA
                elif (h_ionisation if cont else h_excitation) == "drawin":
                    hkind = COLH_DRAWIN
            if kind == 0 and hkind == 0:
                continue
            ci.append(i)
            cj.append(j)
            ck.append(kind)
            chk.append(hkind)
            cf.append(fac)
    return {"col_i": np.array(ci, np.int32), "col_j": np.array(cj, np.int32), "col_kind": np.array(ck, np.int32),
            "col_hkind": np.array(chk, np.int32) if any(chk) else None, "col_fac": np.array(cf, np.float32)}


def _flags(*arrays) -> int:
    for a in arrays:
        if a is not None and not isinstance(a, np.ndarray):
            order_after_torch(a)
            return DEVICE_PTRS
    return 0


def _f64(a):
    if a is None or not isinstance(a, np.ndarray):
        return a
    return np.ascontiguousarray(a, np.float64)


def _f32(a):
    if a is None or not isinstance(a, np.ndarray):
        return a
    return np.ascontiguousarray(a, np.float32)


def _cells(temp, ne, dxi, nh1, lsaha, colliders):
    """The m3d_col_cells_t of the per-cell collision inputs, and the arrays it points into."""
    temp, ne, dxi, nh1, lsaha, colliders = (_f64(a) for a in (temp, ne, dxi, nh1, lsaha, colliders))
    c = ColCells()
    c.temp, c.ne, c.dxi, c.nh1, c.lsaha, c.colliders = (ptr(a) for a in (temp, ne, dxi, nh1, lsaha, colliders))
    c.ncollider = int(colliders.shape[0]) if colliders is not None else 0
    return c, [temp, ne, dxi, nh1, lsaha, colliders]


def collision_nrows(atom: dict) -> int:
    """Rows of a cup buffer: ncol, ncol more with col_hkind, 2 nrec with gencol records."""
    ncol = len(atom["col_i"]) if atom.get("col_i") is not None else 0
    gc = atom.get("gencol")
    return ncol * (2 if atom.get("col_hkind") is not None else 1) + (2 * len(gc["ll"]) if gc is not None else 0)


def collision_rates(atom: dict, temp, ne, e_kT, dxi=None, nh1=None, nstar=None, lsaha=None, colliders=None,
                    out=None):
    """collision_rates' rates [1/s], colscale applied, (collision_nrows, ncell):
    classic_col's upward electron rates, with col_hkind its hydrogen ones (which
    read nh1, the neutral hydrogen ground-level density), then with gencol
    records their upward and downward rates (which read nstar (nlevel, ncell),
    lsaha and, for UP/DN records, colliders (ncollider, ncell))."""
    init()
    st, keep = make_atom(atom)
    cells, keep2 = _cells(temp, ne, dxi, nh1, lsaha, colliders)
    e_kT, nstar = _f64(e_kT), _f64(nstar)
    ncell = int(keep2[0].shape[-1])
    if out is None:
        out = np.zeros((collision_nrows(atom), ncell), np.float64)
    rc = lib().m3d_collision_rates(C.byref(st), C.c_int(ncell), ptr(e_kT), ptr(nstar), C.byref(cells), ptr(out),
                                   C.c_uint(_flags(keep2[0], out)))
    check(rc, "m3d_collision_rates")
    return out


def stateq_update(atom: dict, b, nstar, totn, e_kT, gamma_ij, gamma_ji, temp=None, ne=None, dxi=None, cup=None,
                  nh1=None, lsaha=None, colliders=None, solver: int = LINEQ_NO_PIVOT, max_update: float = 1e2,
                  sor_w: float = 1.0, min_pop_frac: float = 1e-30, conv_pop_floor: float = 0.0, tmax_update: float = 1e7,
                  cswitch: float = 1.0, warp_per_cell: bool = False) -> tuple[dict, np.ndarray]:
    """update_populations over all cells; b (nlevel, ncell) float64 is updated in place.

    Returns (result, lvlerr): maxerr, epos_cell, epos_level, nclamp, ntot,
    nonfinite_cell, the per-level largest change, and team (threads per cell).
    Raises NonFiniteSolution (carrying both) when a cell's solution is not finite.
    warp_per_cell: one warp per cell (M3D_SE_WARP) instead of the library's choice.
    """
    init()
    st, keep = make_atom(atom)
    if isinstance(b, np.ndarray) and (b.dtype != np.float64 or not b.flags.c_contiguous):
        raise M3DError("b must be a C-contiguous float64 array (it is updated in place)")
    nstar, totn, e_kT = _f64(nstar), _f64(totn), _f64(e_kT)
    cup = _f64(cup)
    cells, keep2 = _cells(temp, ne, dxi, nh1, lsaha, colliders)
    gamma_ij, gamma_ji = _f32(gamma_ij), _f32(gamma_ji)
    ncell = int(totn.shape[-1])
    par = SeParams(max_update, sor_w, min_pop_frac, conv_pop_floor, tmax_update, cswitch, int(solver), 0)
    res = SeResult()
    lvlerr = np.zeros(st.nlevel, np.float64)
    rc = lib().m3d_stateq_update(C.byref(st), C.byref(par), C.c_int(ncell), ptr(b), ptr(nstar), ptr(totn),
                                 ptr(e_kT), C.byref(cells), ptr(gamma_ij), ptr(gamma_ji), ptr(cup),
                                 C.c_void_p(lvlerr.ctypes.data), C.byref(res),
                                 C.c_uint(_flags(b, nstar, totn, e_kT) | (SE_WARP if warp_per_cell else 0)))
    out = res.as_dict()
    out["team"] = int(lib().m3d_stateq_team())
    if rc == ENONFINITE:
        from . import last_error
        raise NonFiniteSolution(last_error(), out, lvlerr)
    check(rc, "m3d_stateq_update")
    return out, lvlerr


def ng_accumulate(b, oldb) -> np.ndarray:
    """The Gram matrix d01, d02, d11, d12, d21, d22 and |d0|^2 of ln b over all cells."""
    init()
    b, oldb = _f64(b), _f64(oldb)
    nlevel, ncell = int(b.shape[0]), int(b.shape[1])
    gram = np.zeros(7, np.float64)
    check(lib().m3d_ng_accumulate(C.c_int(ncell), C.c_int(nlevel), ptr(b), ptr(oldb),
                                  C.c_void_p(gram.ctypes.data), C.c_uint(_flags(b, oldb))), "m3d_ng_accumulate")
    return gram


def ng_extrapolate(b, oldb, nstar, totn, a: float, bc: float, max_change: float = 10.0) -> dict:
    """ng_extrapolate in place on b; returns applied, emax, epos_cell, epos_level."""
    init()
    if isinstance(b, np.ndarray) and (b.dtype != np.float64 or not b.flags.c_contiguous):
        raise M3DError("b must be a C-contiguous float64 array (it is updated in place)")
    oldb, nstar, totn = _f64(oldb), _f64(nstar), _f64(totn)
    nlevel, ncell = int(b.shape[0]), int(b.shape[1])
    applied, emax = C.c_int(), C.c_double()
    epc, epl = C.c_longlong(), C.c_int()
    check(lib().m3d_ng_extrapolate(C.c_int(ncell), C.c_int(nlevel), ptr(b), ptr(oldb), ptr(nstar), ptr(totn),
                                   C.c_double(a), C.c_double(bc), C.c_double(max_change), C.byref(applied),
                                   C.byref(emax), C.byref(epc), C.byref(epl), C.c_uint(_flags(b, oldb, nstar, totn))),
          "m3d_ng_extrapolate")
    return {"applied": bool(applied.value), "emax": emax.value, "epos_cell": epc.value, "epos_level": epl.value}


# ---- the host side of Ng (ng_mod.f90:34-229) ----------------------------------------
@dataclass
class NgParams:
    """The &nlte_params gate tunables (ng_mod.f90:34-47)."""

    rate_min: float = 0.5
    rate_tol: float = 0.15
    clamp_max: float = 1e-3
    min_iters_left: int = 3
    cond_min: float = 1e-6
    max_change: float = 10.0
    min_gap: int = 4


@dataclass
class NgState:
    """ng_state_t (ng_mod.f90:61-79); gram vectors are d01, d02, d11, d12, d21, d22."""

    d_cur: np.ndarray = field(default_factory=lambda: np.zeros(6))
    d_done: np.ndarray = field(default_factory=lambda: np.zeros(6))
    s_cur: float = 0.0
    s_done: float = 0.0
    s_prev: float = -1.0
    r: float = -1.0
    r_prev: float = -1.0
    a: float = 0.0
    b: float = 0.0
    nclamp_cur: int = 0
    ntot_cur: int = 0
    nclamp_done: int = 0
    ntot_done: int = 0
    iter_promoted: int = -1
    iter_decided: int = -1
    iter_fired: int = -(2**31 - 1) // 2
    coeff_valid: bool = False
    params: NgParams = field(default_factory=NgParams)

    def condition(self) -> float:
        """ng_condition (ng_mod.f90:88-105): 1 - cos^2 of the angle between d1 and d2."""
        _, _, d11, d12, d21, d22 = self.d_done
        den = d11 * d22 - d12 * d21
        scale = d11 * d22
        return den / scale if scale > 0.0 else 0.0

    def promote(self, it: int) -> None:
        """ng_promote (ng_mod.f90:113-145)."""
        if it <= self.iter_promoted:
            return
        self.iter_promoted = it
        self.d_done = self.d_cur.copy()
        self.s_done = self.s_cur
        self.nclamp_done, self.ntot_done = self.nclamp_cur, self.ntot_cur
        self.d_cur = np.zeros(6)
        self.s_cur = 0.0
        self.nclamp_cur = self.ntot_cur = 0
        if self.s_done > 0.0:
            self.r_prev = self.r
            self.r = math.sqrt(self.s_done / self.s_prev) if self.s_prev > 0.0 else -1.0
            self.s_prev = self.s_done
        self.coeff_valid = False

    def should_fire(self, it: int, err: float, convlim: float) -> tuple[bool, str]:
        """ng_should_fire (ng_mod.f90:153-215): the decision and the declining condition."""
        p = self.params
        if self.s_done <= 0.0 or self.s_prev <= 0.0:
            return False, "no-history"
        if it - self.iter_fired < p.min_gap:
            return False, "min-gap"
        if self.ntot_done <= 0:
            return False, "clamped"
        if self.nclamp_done / self.ntot_done > p.clamp_max:
            return False, "clamped"
        if self.r <= 0.0 or self.r_prev <= 0.0:
            return False, "not-stationary"
        if abs(self.r - self.r_prev) > p.rate_tol * self.r:
            return False, "not-stationary"
        if self.r < p.rate_min:
            return False, "fast-enough"
        if self.r >= 1.0:
            return False, "diverging"
        if abs(err) < convlim * self.r ** (-p.min_iters_left):
            return False, "no-headroom"
        if self.condition() <= p.cond_min:
            return False, "ill-conditioned"
        return True, "FIRE"

    def coefficients(self) -> None:
        """ng_coefficients (ng_mod.f90:221-229)."""
        d01, d02, d11, d12, d21, d22 = self.d_done
        den = d11 * d22 - d12 * d21
        self.a = (d01 * d22 - d02 * d21) / den
        self.b = (d02 * d11 - d01 * d12) / den
        self.coeff_valid = True

    def add_gram(self, gram) -> None:
        """The accumulation of one patch (the critical section of ng_accumulate)."""
        self.d_cur = self.d_cur + np.asarray(gram[:6], np.float64)
        self.s_cur += float(gram[6])

    def count_clamped(self, nclamp: int, ntot: int) -> None:
        """ng_count_clamped (ng_mod.f90:293-302)."""
        self.nclamp_cur += int(nclamp)
        self.ntot_cur += int(ntot)


def _fortran_mod(a: int, p: int) -> int:
    r = abs(a) % abs(p)
    return -r if a < 0 else r


def ng_acceleration(state: NgState, it: int, err: float, convlim: float, b, oldb, nstar, totn,
                    extrapolate: bool = True, ng_step: int = 0, ng_start: int = 0) -> dict:
    """atom_type%ng_acceleration (atom_mod.f90:2469-2548) for one set of cells.

    b (nlevel, ncell) and oldb (3, nlevel, ncell), the iterates n1, n2, n3 that
    normalize_profiles shifts, stay on the device when they are CUDA tensors.
    Returns emax, epos_cell, epos_level, applied and the gate's reason.
    """
    out = {"emax": 0.0, "epos_cell": -1, "epos_level": -1, "applied": False, "reason": "decided"}
    state.promote(it)
    if it > state.iter_decided:
        state.iter_decided = it
        if ng_step > 0:
            fire = _fortran_mod(it - ng_start, ng_step) == 1 and state.s_done > 0.0
            out["reason"] = "FIRE" if fire else "off-cycle"
        else:
            fire, out["reason"] = state.should_fire(it, err, convlim)
        if fire:
            state.coefficients()
            state.iter_fired = it
    if state.coeff_valid and state.iter_fired == it and extrapolate:
        r = ng_extrapolate(b, oldb, nstar, totn, state.a, state.b, state.params.max_change)
        out.update(r)
    if it >= 3 and state.iter_fired != it and oldb is not None:
        state.add_gram(ng_accumulate(b, oldb))
    return out


def shift_oldb(oldb, b) -> None:
    """The history shift of normalize_profiles (atom_mod.f90:423-429): n1 <- n2 <- n3 <- b."""
    oldb[0] = oldb[1]
    oldb[1] = oldb[2]
    oldb[2] = b

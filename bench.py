"""Throughput of the OpenMULTI3D LTE output pass on B200.

Workload (the 3D LTE synthesis configuration): a 240^3 seeded synthetic cube in 10
depth slabs of 24 planes, 500 lines in 5000-5020 A, 4000 frequencies uniform in
ln(lambda) split into windows of --nf frequencies, 13 output rays (Lobatto 4x4),
rotate_array + long_char_quadratic.  One step is one frequency window for every
ray: line opacity, transfer units, the slab-by-slab sweep, emergent intensity and
flux.  Metric: Gpt*nu*ray/s = 1e-9 * rays * cells * frequencies / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--nf NF] [--impl reference]

Ranks (torchrun) each take their own frequency windows, spread over the band: the
windows are independent (weak scaling, no data-path collective).  --impl reference times the
CPU restatement of the reference on this host's cores on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "formal-solve Gpt*nu*ray/s on 1 B200, FP32 vs FP64 path at <=1e-4 flux error"
UNIT = "Gpt*nu*ray/s"
NFREQ_TOTAL = 4000
REF_NCOLS = 8          # the CPU sample: 8 x 8 columns of the cube, full depth


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=8)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--nf", type=int, default=32)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-ali", action="store_true", help="skip the NLTE measurements (3D window, batched columns)")
    p.add_argument("--no-optab", action="store_true", help="skip the sampled opacity table measurement")
    p.add_argument("--no-c0", action="store_true", help="skip the 1D LTE synthesis measurement")
    p.add_argument("--no-c4", action="store_true", help="skip the differentiable (adjoint) measurement")
    p.add_argument("--cube", type=int, default=240, help="cube edge (240 = the configuration; smaller for profiling)")
    # single cases for timing and profiling one kernel family (no JSON line)
    p.add_argument("--case", default="c1",
                   choices=["c1", "ali-window", "ali-columns", "optab", "c2", "batched", "continuum", "c0"],
                   help="c1: the headline (default); the others run one seeded NLTE or table case and print "
                        "per-iteration times")
    p.add_argument("--n", type=int, default=64, help="ali-window / optab / continuum: cube edge")
    p.add_argument("--ncol", type=int, default=1024, help="ali-columns: columns")
    p.add_argument("--nbound", type=int, default=20, help="ali-*: bound levels of the model atom")
    p.add_argument("--nline", type=int, default=60, help="ali-*: bound-bound transitions of the model atom")
    p.add_argument("--every", type=int, default=8, help="ali-window: the window holds every k-th transition")
    p.add_argument("--nwin", type=int, default=8, help="ali-columns: frequency windows")
    p.add_argument("--iters", type=int, default=2, help="ali-* / optab: iterations")
    p.add_argument("--no-graph", action="store_true", help="ali-columns: direct launches instead of the graph")
    p.add_argument("--per-point", action="store_true",
                   help="ali-columns: the per-point kernels instead of the fused column sweep")
    p.add_argument("--only", choices=["sample", "ll"], default=None, help="optab: one sampler")
    return p.parse_args()


def _workload(nf, n=240):
    return {"workload": f"c1 3D LTE synthesis: {n}^3 cube in 10 slabs of {n // 10} planes, 500 lines 5000-5020 A, "
                        f"4000 frequencies in windows of {nf}, 13 rays (Lobatto 4x4), rotate_array + "
                        "long_char_quadratic; one step = one frequency window, all rays",
            "cells": n ** 3, "rays": 13, "nf_window": nf, "nf_total": NFREQ_TOTAL, "slabs": 10,
            "l2": "inputs larger than L2 (0.7 GB atmosphere + 3.5 GB transfer units per window)"}


def _make_inputs(nf, n=240):
    from dispatch_b200 import synth
    atm, _, _, vec, wmu = synth.lte_config("c1", nf=nf, window=0, size=None if n == 240 else n)
    llam_all, nu_all = synth.frequency_grid(5000.0, 5020.0, NFREQ_TOTAL)
    return atm, llam_all, nu_all, vec, wmu


def _window(llam_all, nu_all, nf, w):
    nwin = nu_all.size // nf
    w = w % nwin
    sl = slice(w * nf, (w + 1) * nf)
    return np.ascontiguousarray(nu_all[sl]), np.ascontiguousarray(llam_all[sl])


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return None


# Figures of one ncu capture of the 48^3 case of the same configuration (one launch of
# each kernel; the command is in the summaries under profiles/).
#  k_quad_rot_column2: DRAM bytes per cell and frequency of a launch (28,360,192 B read
#    for 110,592 cells x 32 frequencies), against 8 B algorithmic (chi and Snu once).
#  k_lte_opacity_units_lane<32>: warp instructions per (cell, line), the mean over the
#    104 launches of the 8 timed windows x 13 rays (79,401,861,582 for 110,592 cells x
#    500 lines each; 13.0-14.8 per launch as the windows' line loads differ), which
#    scales a full launch's count by its cells and lines; DRAM bytes per cell: 49.9 B
#    read (measured, window 0) plus the chi and
#    Snu it writes, 8 B per frequency (the small case's 28 MB of output stayed in L2,
#    a full launch's 3.5 GB cannot).
NCU_SWEEP_DRAM_BYTES_PER_CELL_FREQ = 8.013
#  k_quad_rot_column2: warp instructions per (cell, frequency) of a launch
#    (21,865,784 for 110,592 cells x 32 frequencies)
NCU_SWEEP_WARP_INST_PER_CELL_FREQ = 21865784 / (110592 * 32)
NCU_OPACITY_WARP_INST_PER_CELL_LINE = 79401861582 / (104 * 110592 * 500)
NCU_OPACITY_DRAM_READ_BYTES_PER_CELL = 5516032 / 110592
#  k_continuum: warp instructions per cell of a launch of the continuum case (250
#    frequencies, fourteen components; 904,826,466 for 110,592 cells)
NCU_CONTINUUM_WARP_INST_PER_CELL = 904826466 / 110592


def _subcube(atm, n):
    nx, ny, nz = atm["nx"], atm["ny"], atm["nz"]

    def cut(a):
        return np.ascontiguousarray(a.reshape(nz, ny, nx)[:, :n, :n]).ravel()

    sub = dict(atm)
    sub["nx"] = sub["ny"] = n
    for k in ("temp", "chi_c", "vx", "vy", "vz", "e_kT", "ne", "tothi", "stark_pe"):
        sub[k] = cut(atm[k])
    sub["species"] = [{k: (cut(v) if k in ("inv_df", "vbar2", "lnbase") else v) for k, v in sp.items()}
                      for sp in atm["species"]]
    return sub


def _cells(atm, lo, hi):
    """The cells lo:hi of an atmosphere as a row of independent cells (the opacity
    stage is per cell)."""
    sub = {"nx": hi - lo, "ny": 1, "nz": 1, "slab_nz": [1]}
    for k in ("temp", "chi_c", "vx", "vy", "vz", "e_kT", "ne", "tothi", "stark_pe"):
        sub[k] = np.ascontiguousarray(atm[k][lo:hi])
    sub["species"] = [{k: (np.ascontiguousarray(v[lo:hi]) if k in ("inv_df", "vbar2", "lnbase") else v)
                       for k, v in sp.items()} for sp in atm["species"]]
    return sub


def _ref_units(args):
    sub, nu, llam, v = args
    from oracle import pipeline as P
    return P.transfer_units(sub, nu, llam, v)


def _ref_sweep(args):
    sub, chi, S, v = args
    from oracle import pipeline as P
    return P.column_sweep(sub, chi, S, v)


class CpuReference:
    """The oracle (the C restatement of the reference, built -O3 -march=x86-64-v3 as
    the reference's release build) on every host core: the opacity stage split over
    (ray, chunk of cells), then the column sweep of every ray, over an ncols x ncols
    block of columns of the cube (full depth, all slabs), one window, all rays."""

    def __init__(self, atm, vec, wmu, ncols):
        import multiprocessing as mp
        self.sub = _subcube(atm, ncols)
        self.vec, self.wmu, self.ncols = vec, wmu, ncols
        self.cores = os.cpu_count() or 1
        ncell = self.sub["nx"] * self.sub["ny"] * self.sub["nz"]
        nchunk = max(1, self.cores)
        edges = np.linspace(0, ncell, nchunk + 1).astype(int)
        self.chunks = [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]
        self.parts = [_cells(self.sub, a, b) for a, b in self.chunks]
        self.pool = mp.get_context("spawn").Pool(self.cores)
        self.work = vec.shape[0] * ncell

    def step(self, nu, llam):
        from oracle import oracle as O
        nray = self.vec.shape[0]
        tasks = [(part, nu, llam, self.vec[r]) for r in range(nray) for part in self.parts]
        res = self.pool.map(_ref_units, tasks, chunksize=1)
        k, sweeps = 0, []
        for r in range(nray):
            chi = np.concatenate([res[k + i][0] for i in range(len(self.parts))])
            S = np.concatenate([res[k + i][1] for i in range(len(self.parts))])
            k += len(self.parts)
            sweeps.append((self.sub, chi, S, self.vec[r]))
        tops = self.pool.map(_ref_sweep, sweeps, chunksize=1)
        return O.save_intensity(nu, np.stack(tops).astype(np.float32), self.wmu)[1]

    def close(self):
        self.pool.close()
        self.pool.join()

    def describe(self, nf, seconds):
        return (f"{self.ncols}x{self.ncols} columns x {self.sub['nz']} planes ({len(self.sub['slab_nz'])} slabs) x "
                f"{nf} frequencies x {self.vec.shape[0]} rays of the same cube and windows; opacity over "
                f"(ray, {len(self.parts)} cell chunks), sweep per ray, {self.cores} processes; "
                f"C restatement of the reference (-O3 -march=x86-64-v3), {seconds:.1f} s")


def _timed_windows(rank: int, steps_total: int, nwin: int) -> list[int]:
    """The windows a rank's steps take: spread over the band (stride 37, coprime with
    the 125 windows of 32 frequencies), each rank its own, the same on both arms."""
    return [((rank * steps_total + i) * 37) % nwin for i in range(steps_total)]


def run_reference(a):
    """The reference arm: the CPU restatement on all host cores, the same windows as
    the device arm times, a bounded block of columns per step."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    atm, llam_all, nu_all, vec, wmu = _make_inputs(a.nf)
    steps_total = a.warmup + a.steps
    wins = _timed_windows(0, steps_total, NFREQ_TOTAL // a.nf)
    ref = CpuReference(atm, vec, wmu, ncols=REF_NCOLS)
    for i in range(a.warmup):
        ref.step(*_window(llam_all, nu_all, a.nf, wins[i]))
    t0 = time.perf_counter()
    for i in range(a.warmup, steps_total):
        ref.step(*_window(llam_all, nu_all, a.nf, wins[i]))
    dt = (time.perf_counter() - t0) / a.steps
    ref.close()
    value = ref.work * a.nf / dt / 1e9
    sample = ref.describe(a.nf, dt * a.steps)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": _workload(a.nf),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _nlte_ali(steps=2):
    """The ALI window of the 3D NLTE configuration, measured beside the headline: the
    120^3 cube, the 20-level atom, a frequency window holding 10 of its 80 transitions
    (every eighth: 8 lines and 2 continua, 250 frequencies), both hemispheres of the
    Lobatto 4x4 directions (26).  A sweep is one ALI iteration's formal solutions with
    the opacities, J, PsiJ and rate integrals of every direction; the update is the
    FP64 statistical equilibrium of all 1.728 M cells (fused collision rates, the Ng
    gate).  Device-resident inputs; CUDA events on torch's stream."""
    import torch

    import dispatch_b200 as m
    from dispatch_b200 import ali
    cube, atom, win, vec, wts = ali.cube_problem("c2", transitions=list(range(0, 80, 8)))
    A = ali.AliWindow(cube, atom, win, vec, wts)
    A.sweep()
    A.iter = 1
    A.update()
    cur = torch.cuda.current_stream()
    sw, up, n0 = [], [], m.launch_count()
    for _ in range(steps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(cur)
        A.sweep()
        e1.record(cur)
        A.iter += 1
        rec = A.update()
        e2.record(cur)
        torch.cuda.synchronize()
        sw.append(e0.elapsed_time(e1))
        up.append(e1.elapsed_time(e2))
    pts = A.points()
    sweep_ms = float(np.median(sw))
    out = {"workload": "c2 3D NLTE ALI window: 120^3 cube, 20-level atom, 10 of 80 transitions (8 lines, "
                       "2 continua; 250 frequencies), 26 directions (Lobatto 4x4, both hemispheres), "
                       "short_char with split rates ('largest'), lineq_no_pivot",
           "unit": UNIT, "value": pts / (sweep_ms / 1e3) / 1e9, "sweep_ms": sweep_ms,
           "update_ms": float(np.median(up)), "cells_per_s_update": A.ncell / (float(np.median(up)) / 1e3),
           "ray_pt_nu_per_sweep": pts, "gpu_launches_per_iteration": (m.launch_count() - n0) // steps,
           "maxerr_last": rec["maxerr"], "data": "synthetic (seeded grey cube, seeded model atom)"}
    del A
    torch.cuda.empty_cache()
    return out


def _nlte_batched(steps=2):
    """The batched 1.5D NLTE configuration, measured beside the headline: 4096 columns
    of 60-256 cells from a seeded 64 x 64 x 256 cube, three abundance variants
    (0, +-0.2 dex) packed as further columns (1.94 M cells), the 21-level atom (80
    transitions, 8 windows, 2000 frequencies) and the 61-level atom (240 transitions,
    24 windows, 6000 frequencies), Radau 2 directions and their mirror (4).  Each
    atom's sweep is one CUDA-graph replay of its column plan; an ALI iteration is
    both sweeps and both atoms' statistical-equilibrium updates."""
    import torch

    import dispatch_b200 as m
    from dispatch_b200 import ali, synth
    cols = synth.column_set(3, ncol=4096, depth=(60, 256), nz=256, nxy=64, variants=(0.0, 0.2, -0.2))
    vec, wts = synth.radau_rays(2, 1, jnu_weights=True)
    plans = []
    for nb, nl in ((20, 60), (60, 180)):
        atom = synth.model_atom(3, nbound=nb, nline=nl)
        nrad = len(atom["ti"])
        nwin = max(1, nrad // 10)
        wins = [synth.atom_window(atom, seed=3, transitions=list(range(k, nrad, nwin))) for k in range(nwin)]
        plans.append(ali.AliColumns(cols, atom, wins, vec[:, 2].copy(), wts, params=ali.AliParams(convlim=1e-9)))
    for A in plans:
        A.sweep()
    cur = torch.cuda.current_stream()
    sw, up, n0 = [], [], m.launch_count()
    for _ in range(steps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(cur)
        for A in plans:
            A.iter += 1
            A.update()
        e1.record(cur)
        for A in plans:
            A.sweep()
        e2.record(cur)
        torch.cuda.synchronize()
        up.append(e0.elapsed_time(e1))
        sw.append(e1.elapsed_time(e2))
    pts = sum(A.points() for A in plans)
    sweep_ms, update_ms = float(np.median(sw)), float(np.median(up))
    shapes = [A.shape for A in plans]
    launches = (m.launch_count() - n0) // steps
    for A in plans:
        A.close()
    # the same sweeps by the per-point kernels (opacity, column solver, rate sums as
    # separate launches through HBM), for comparison: one warm-up and one timed sweep
    pp = []
    for nb, nl in ((20, 60), (60, 180)):
        atom = synth.model_atom(3, nbound=nb, nline=nl)
        nrad = len(atom["ti"])
        nwin = max(1, nrad // 10)
        wins = [synth.atom_window(atom, seed=3, transitions=list(range(k, nrad, nwin))) for k in range(nwin)]
        A = ali.AliColumns(cols, atom, wins, vec[:, 2].copy(), wts, params=ali.AliParams(convlim=1e-9), fused=False)
        A.sweep()
        e0, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(2))
        torch.cuda.synchronize()
        e0.record(cur)
        A.sweep()
        e1.record(cur)
        torch.cuda.synchronize()
        pp.append(e0.elapsed_time(e1))
        A.close()
        del A
        torch.cuda.empty_cache()
    out = {"workload": "batched 1.5D NLTE: 4096 columns of 60-256 cells (seeded 64x64x256 cube), 3 abundance "
                       "variants (1.94 M cells), 21-level atom (2000 frequencies, 8 windows) and 61-level atom "
                       "(6000 frequencies, 24 windows), Radau 2 + mirror (4 directions), long_char_linear along "
                       "each column with split rates; each atom's sweep one CUDA graph replay",
           "unit": UNIT, "value": pts / (sweep_ms / 1e3) / 1e9, "sweep_ms": sweep_ms, "update_ms": update_ms,
           "iteration_ms": sweep_ms + update_ms, "ray_pt_nu_per_iteration": pts,
           "graph_launches_per_iteration": launches,
           "plan_shapes_autotuned": shapes, "cells": plans[0].ncell,
           "per_point_sweep_ms": float(sum(pp)),
           "per_point_value": pts / (sum(pp) / 1e3) / 1e9,
           "data": "synthetic (seeded grey cube, seeded model atoms)"}
    del plans
    torch.cuda.empty_cache()
    return out


def _continuum(steps=5, warmup=3, n=120, sm_mhz=None):
    """The continuum opacity of one window (HOP's continuum_opacities): the 120^3
    cube's 1.73 M cells, 250 frequencies in 3500-12000 A, fourteen absdat-like
    components of every kind (synth.continuum_case), the H rest, electron and
    Rayleigh scattering; inputs resident on the device, CUDA events on torch's
    stream.  Beside it the C restatement on one core over 2000 cells of the same
    case."""
    import torch

    from dispatch_b200 import synth
    from dispatch_b200.continuum import continuum_opacities
    ncell, nlam = n**3, 250
    comps, lam, nu, cells = synth.continuum_case(ncell=ncell, nlam=nlam)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dc = {k: (dev(v) if isinstance(v, np.ndarray) else v) for k, v in cells.items()}
    dcomps = [{k: (dev(v) if k in ("n", "n2", "part", "level_n", "level_w") else v) for k, v in c.items()}
              for c in comps]
    cur = torch.cuda.current_stream()
    for _ in range(warmup):
        continuum_opacities(dcomps, lam, nu, dc)
    ts = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(cur)
        xh, sg = continuum_opacities(dcomps, lam, nu, dc)
        e1.record(cur)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    # algorithmic bytes: xhat and sigma written, the cells' EOS state and densities read
    ncarr = 11 + sum(sum(1 for k in ("n", "n2", "part", "level_n", "level_w") if c.get(k) is not None) for c in comps)
    nbytes = 8.0 * nlam * ncell + 8.0 * ncarr * ncell
    peaks = _peaks() or {}
    peak = peaks.get("hbm_gbs", 6650.0)
    from oracle import continuum as oc
    sub = 2000
    sc = {k: (v[:sub] if isinstance(v, np.ndarray) else v) for k, v in cells.items()}
    scomps = [{k: (v[:sub] if k in ("n", "n2", "part", "level_n", "level_w") else v) for k, v in c.items()}
              for c in comps]
    t0 = time.perf_counter()
    oc.continuum_opacities(scomps, lam, nu, sc)
    dt = time.perf_counter() - t0
    del xh, sg, dc, dcomps
    torch.cuda.empty_cache()
    # bound by instruction issue like the line opacity: 148 SMs x 4 schedulers x one
    # warp instruction per cycle, the instructions per launch scaled from the ncu count
    # of the 48^3 case by cells
    issue_peak = 148 * 4 * (sm_mhz or 1965.0) / 1e3
    inst = NCU_CONTINUUM_WARP_INST_PER_CELL * ncell
    issue = {"kernel": "k_continuum", "bound": "issue", "achieved": inst / (ms / 1e3) / 1e9, "peak": issue_peak,
             "unit": "G warp-instructions/s", "frac": inst / (ms / 1e3) / 1e9 / issue_peak,
             "warp_instructions_per_launch": inst,
             "peak_source": "148 SMs x 4 issue slots x " + ("sampled SM clock" if sm_mhz else "max SM clock")}
    return {"workload": f"continuum opacity of one window: {ncell / 1e6:.2f} M cells ({n}^3), {nlam} frequencies "
                        "3500-12000 A, 14 absdat-like components of every kind (2 H BF levels under occupation "
                        "probabilities), H rest, electron + Rayleigh scattering",
            "unit": "Gpt*nu/s", "ms": ms, "value": ncell * nlam / (ms / 1e3) / 1e9,
            "achieved_gbs": nbytes / (ms / 1e3) / 1e9, "peak_gbs": peak, "frac": nbytes / (ms / 1e3) / 1e9 / peak,
            "roofline_issue": issue,
            "cpu_baseline": {"value": sub * nlam / dt / 1e9, "unit": "Gpt*nu/s", "cores": 1, "kind": "port",
                             "sample": f"{sub} cells of the same case, the C restatement on one core, {dt:.2f} s"},
            "data": "synthetic (seeded EOS state and tables)"}


def _optab(steps=5, warmup=3):
    """The sampled opacity tables (HOP/optab_mod.f90), measured beside the headline:
    2.1 M cells of a seeded 128^3 cube and one window of 256 frequencies at R = 1e5,
    the tables built as the reference builds them for a window: the background
    table on the window's own wavelengths (every query on a node), the line-list
    table on them padded for the largest Doppler shift.  sample_interpolate sets
    back and scat; sample_interpolate_ll with the cube's projected velocities adds
    into xhat, ehat and chi_scat.  Device-resident inputs, outputs larger than L2;
    CUDA events on torch's stream.  Algorithmic bytes per (frequency, cell): 8
    written by sample_interpolate, 24 read and written by sample_interpolate_ll;
    per cell 20 and 24 read.  The tables (a few tens of MB) stay in L2."""
    import torch

    import dispatch_b200 as m
    from dispatch_b200 import synth
    from dispatch_b200.optab import SampleOptab
    c = synth.optab_cells(7, 128, 128, 128)
    ncell, nf = c["temp"].size, 256
    lam_q, bg, ll = synth.window_tables(8, c["temp"], c["ne"], c["vproj"], nf=nf)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    T, N, X, V = dev(c["temp"]), dev(c["ne"]), dev(c["chi500"]), dev(c["vproj"])
    q = dev(lam_q)
    tb, tl = SampleOptab.from_dict(bg), SampleOptab.from_dict(ll)
    back = torch.empty((ncell, nf), dtype=torch.float32, device="cuda")
    scat = torch.empty_like(back)
    xh, eh, cs = torch.zeros_like(back), torch.zeros_like(back), torch.zeros_like(back)
    cur = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(warmup):
            fn()
        ts = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(cur)
            fn()
            e1.record(cur)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    n0 = m.launch_count()
    t_s = timed(lambda: tb.interpolate(T, N, X, q, back, scat))
    t_l = timed(lambda: tl.interpolate_ll(T, N, X, xh, eh, q, V, cs))
    launches = (m.launch_count() - n0) // (2 * (steps + warmup))
    peaks = _peaks() or {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    pts = ncell * nf
    out = {"workload": "sampled opacity tables: 2.1 M cells (seeded 128^3 cube), one window of 256 frequencies at "
                       "R = 1e5; background table %d x %d x %d nodes on the window's wavelengths (value + "
                       "scattering), line-list table %d x %d x %d padded for the Doppler shifts"
                       % (tb.nnu, tb.ntemp, tb.nne, tl.nnu, tl.ntemp, tl.nne),
           "unit": "Gpt*nu/s", "launches_per_call": launches, "data": "synthetic (seeded cube, seeded tables)"}
    for name, t, per_pt, per_cell in (("sample_interpolate", t_s, 8, 20), ("sample_interpolate_ll", t_l, 24, 24)):
        gbs = (per_pt * pts + per_cell * ncell) / (t / 1e3) / 1e9
        out[name] = {"ms": t, "value": pts / (t / 1e3) / 1e9, "achieved_gbs": gbs, "peak_gbs": hbm,
                     "frac": gbs / hbm, "peak_kind": "measured" if peaks else "fallback"}
    # the oracle on a bounded sample of the same cells, one host thread
    from oracle import optab as oopt
    k = 4096
    t0 = time.perf_counter()
    oopt.sample(bg, c["temp"][:k], c["ne"][:k], c["chi500"][:k], lam_q)
    out["cpu_baseline"] = {"value": k * nf / (time.perf_counter() - t0) / 1e9, "unit": "Gpt*nu/s", "cores": 1,
                           "kind": "port", "sample": f"{k} cells x {nf} frequencies, including the node slopes"}
    tb.close()
    tl.close()
    del back, scat, xh, eh, cs
    torch.cuda.empty_cache()
    return out


def _c4(m, nwin=2):
    """The differentiable 3D LTE configuration, measured beside the headline: the
    96x96x128 seeded cube (8 slabs of 16 planes), ten species of 100 lines in
    6000-6050 A, windows of 32 of the 8000 frequencies, 13 rays.  Per window: the FP32
    forward pass (m3d_lte_synthesis), its adjoint (m3d_lte_synthesis_adjoint: the
    gradients with respect to temperature, e_kT, the Doppler factors, lnbase and every
    line's gpref), and the plain FP64 forward.  Device-resident inputs; CUDA events on
    torch's stream."""
    import torch
    from dispatch_b200 import synth
    atm, _, _, vec, wmu, raw = synth.lte_config_c4()
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    datm = {k: (dev(v) if isinstance(v, np.ndarray) else v) for k, v in atm.items()}
    datm["species"] = [{k: dev(v) for k, v in sp.items()} for sp in atm["species"]]
    ncell = atm["nx"] * atm["ny"] * atm["nz"]
    nline = sum(len(sp["llam0"]) for sp in atm["species"])
    wins = [nwin_i * 97 % 250 for nwin_i in range(1, nwin + 1)]
    cur = torch.cuda.current_stream()
    rng = np.random.default_rng(5)
    g_flux = dev(rng.uniform(0.5, 1.5, 32).astype(np.float32))
    grads = {"temp": torch.zeros(ncell, device="cuda"), "chi_c": torch.zeros(ncell, device="cuda"),
             "e_kT": torch.zeros(ncell, device="cuda"), "inv_df": torch.zeros((10, ncell), device="cuda"),
             "lnbase": torch.zeros((10, ncell), device="cuda"), "gpref": torch.zeros(nline, device="cuda")}
    m.set_stream(cur.cuda_stream or 1)

    def timed(fn):
        fn(wins[0])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        for w in wins:
            fn(w)
        e1.record(cur)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / len(wins)

    def win(w):
        return tuple(dev(x) for x in _window(raw["llam_all"], raw["nu_all"], 32, w))

    dw = {w: win(w) for w in wins}
    fwd = timed(lambda w: m.lte_synthesis(datm, dw[w][0], dw[w][1], vec, wmu, device=True))
    bwd = timed(lambda w: m.lte_synthesis_adjoint(datm, dw[w][0], dw[w][1], vec, wmu, g_flux, device=True,
                                                 grads=grads))
    f64 = timed(lambda w: m.lte_synthesis(datm, dw[w][0], dw[w][1], vec, wmu, device=True, fp64=True))
    m.profile_enable(True)
    m.lte_synthesis_adjoint(datm, dw[wins[0]][0], dw[wins[0]][1], vec, wmu, g_flux, device=True, grads=grads)
    stages = {"opacity_ms": m.profile_read(m.STAGE_OPACITY)[0], "sweep_ms": m.profile_read(m.STAGE_SOLVE)[0]}
    m.profile_enable(False)
    work = vec.shape[0] * ncell * 32
    out = {"workload": "c4 differentiable 3D LTE: 96x96x128 cube in 8 slabs, 10 species x 100 lines 6000-6050 A, "
                       "windows of 32 of 8000 frequencies, 13 rays; forward, adjoint (d/dT, e_kT, Doppler "
                       "factors, lnbase, every line's gpref) and the plain FP64 forward per window",
           "unit": UNIT, "windows_timed": wins, "ray_pt_nu_per_window": work,
           "forward_fp32": {"ms": fwd, "value": work / (fwd / 1e3) / 1e9},
           "adjoint_fp32": {"ms": bwd, "value": work / (bwd / 1e3) / 1e9},
           "forward_plus_adjoint_fp32": {"ms": fwd + bwd, "value": work / ((fwd + bwd) / 1e3) / 1e9},
           "forward_fp64_plain": {"ms": f64, "value": work / (f64 / 1e3) / 1e9},
           "fp32_forward_plus_adjoint_over_fp64_forward": f64 / (fwd + bwd),
           "adjoint_stages": stages,
           "gradients_finite": bool(all(torch.isfinite(v).all() for v in grads.values())),
           "data": "synthetic (seeded cube, ten-species random line list)"}
    del datm, grads
    torch.cuda.empty_cache()
    return out


def _c0(m, a):
    """The 1D plane-parallel LTE synthesis configuration, measured beside the headline:
    80 depths, 2000 lines in 5000-5100 A, all 20000 frequencies in 625 windows of 32,
    5 Gauss-Legendre rays, long_char_quadratic, FP32 and the plain FP64 path; the CPU
    restatement on a bounded sample of the windows.  All 625 windows in one
    m3d_lte_synthesis_windows call over the device-resident column (one opacity
    launch per ray for every window); beside it the same windows one call each."""
    import torch
    from dispatch_b200 import synth
    atm, _, _, vec, wmu = synth.lte_config("c0", nf=32, window=0)
    llam_all, nu_all = synth.frequency_grid(5000.0, 5100.0, 20000)
    nwin = 20000 // 32
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    datm = {k: (dev(v) if isinstance(v, np.ndarray) else v) for k, v in atm.items()}
    datm["species"] = [{k: dev(v) for k, v in sp.items()} for sp in atm["species"]]
    wins = [tuple(dev(x) for x in _window(llam_all, nu_all, 32, w)) for w in range(nwin)]
    nu_b, llam_b = dev(nu_all[:nwin * 32].reshape(nwin, 32)), dev(llam_all[:nwin * 32].reshape(nwin, 32))
    cur = torch.cuda.current_stream()
    out = {"workload": "c0 1D LTE synthesis: 80 depths, 2000 lines 5000-5100 A, 20000 frequencies (625 windows "
                       "of 32), 5 Gauss rays, long_char_quadratic", "unit": UNIT,
           "ray_pt_nu": 5 * 80 * 20000, "data": "synthetic (grey column, random line list)"}
    flux = {}
    for fp64 in (False, True):
        for _ in range(3):
            m.lte_synthesis_windows(datm, nu_b, llam_b, vec, wmu, device=True, fp64=fp64)
        ts = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(cur)
            fl = m.lte_synthesis_windows(datm, nu_b, llam_b, vec, wmu, device=True, fp64=fp64)[1]
            e1.record(cur)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        flux[fp64] = fl.double()
        out["fp64" if fp64 else "fp32"] = {"ms": ms, "value": out["ray_pt_nu"] / (ms / 1e3) / 1e9}
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    out["max_rel_flux_err_fp32_vs_fp64"] = float((torch.abs(flux[False] - flux[True]) / flux[True]).max().item())
    # the same windows one m3d_lte_synthesis call each (FP32), and their flux against the batch's
    for nu_d, llam_d in wins[:3]:
        m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(cur)
    fl = [m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True)[1] for nu_d, llam_d in wins]
    e1.record(cur)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["fp32_one_call_per_window"] = {"ms": ms, "value": out["ray_pt_nu"] / (ms / 1e3) / 1e9,
                                       "flux_equals_batch": bool(torch.equal(torch.cat(fl).double(), flux[False]))}
    # the CPU restatement: every 25th window, one process per window over all cores
    import multiprocessing as mp
    sample = list(range(0, nwin, 25))
    tasks = [(atm, *_window(llam_all, nu_all, 32, w), vec, wmu) for w in sample]
    cores = min(os.cpu_count() or 1, len(tasks))
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_c0_task, tasks[:cores])
        t0 = time.perf_counter()
        pool.map(_c0_task, tasks, chunksize=1)
        dt = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": 5 * 80 * 32 * len(sample) / dt / 1e9, "unit": UNIT, "cores": cores,
                           "kind": "port", "sample": f"{len(sample)} of the 625 windows (every 25th), one process "
                                                     f"per window, C restatement (-O3 -march=x86-64-v3), {dt:.1f} s"}
    return out


def _c0_task(args):
    atm, nu, llam, vec, wmu = args
    from oracle import pipeline as P
    return P.lte_synthesis(atm, nu, llam, vec, wmu)[1]


def run_b200(a):
    import torch
    import torch.distributed as dist

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    import dispatch_b200 as m

    m.init(local)
    stream = torch.cuda.current_stream()
    # the library's work on the stream the timing events are recorded on (torch's
    # default stream is the legacy one, named by cudaStreamLegacy = 0x1)
    m.set_stream(stream.cuda_stream or 1)
    nf = a.nf
    atm, llam_all, nu_all, vec, wmu = _make_inputs(nf, a.cube)
    ncell = atm["nx"] * atm["ny"] * atm["nz"]
    nray = wmu.size
    work_per_step = nray * ncell * nf

    def to_dev(x):
        return torch.from_numpy(np.ascontiguousarray(x)).to(f"cuda:{local}")

    datm = {k: (to_dev(v) if isinstance(v, np.ndarray) else v) for k, v in atm.items()}
    datm["species"] = [{k: to_dev(v) for k, v in sp.items()} for sp in atm["species"]]
    nwin = NFREQ_TOTAL // nf
    steps_total = a.warmup + a.steps
    wins = _timed_windows(rank, steps_total, nwin)
    dwin = [tuple(to_dev(x) for x in _window(llam_all, nu_all, nf, w)) for w in wins]

    def step(i):
        nu_d, llam_d = dwin[i]
        return m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True)

    for i in range(a.warmup):
        step(i)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    n0 = m.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(a.warmup, steps_total):
            step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = m.launch_count() - n0
    ms = ev0.elapsed_time(ev1)
    if ws > 1:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = ws * a.steps * work_per_step / (ms / 1e3) / 1e9
    clocks = clk.summary()

    # stage times and the kernels' rooflines (library CUDA events on its stream): the
    # first timed window alone (the FP64 pass's window), then every timed window again,
    # so the per-step stage times average the windows the timed steps ran
    m.profile_enable(True)
    step(a.warmup)
    op1_ms, _ = m.profile_read(m.STAGE_OPACITY)
    sv1_ms, _ = m.profile_read(m.STAGE_SOLVE)
    m.profile_enable(True)
    for i in range(a.warmup, steps_total):
        step(i)
    op_tot, op_n = m.profile_read(m.STAGE_OPACITY)
    sv_tot, sv_n = m.profile_read(m.STAGE_SOLVE)
    rd_tot, rd_n = m.profile_read(m.STAGE_REDUCE)
    m.profile_enable(False)
    op_ms, sv_ms, rd_ms = op_tot / a.steps, sv_tot / a.steps, rd_tot / a.steps
    peaks = _peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    peak_kind = "measured" if peaks else "fallback"
    # the step's dominant kernel, the line opacity, is bound by instruction issue (its
    # DRAM traffic is a few bytes per cell): its roofline is the issue rate of the SMs,
    # 148 SMs x 4 schedulers x one warp instruction per cycle at the SM clock sampled
    # during the timed region; its instructions per launch are the ncu count of the
    # small case per (cell, line), times this launch's cells and lines
    nline = sum(len(sp["llam0"]) for sp in atm["species"])
    sm_hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    issue_peak = 148 * 4 * sm_hz / 1e9
    op_launch_s = op_tot / op_n / 1e3 if op_n else None
    inst = (NCU_OPACITY_WARP_INST_PER_CELL_LINE * ncell * nline) if NCU_OPACITY_WARP_INST_PER_CELL_LINE else None
    op_achieved = inst / op_launch_s / 1e9 if (inst and op_launch_s) else None
    roofline = {"kernel": "k_lte_opacity_units_lane<32> (line opacity + transfer units, one ray)", "bound": "issue",
                "achieved": op_achieved, "peak": issue_peak, "unit": "G warp-instructions/s",
                "frac": op_achieved / issue_peak if op_achieved else None,
                "traffic": (NCU_OPACITY_DRAM_READ_BYTES_PER_CELL + 8.0 * nf) * ncell,
                "warp_instructions_per_launch": inst, "share_of_step": op_ms / (op_ms + sv_ms + rd_ms) if op_ms else None,
                "peak_source": "148 SMs x 4 issue slots x sampled SM clock",
                "hbm_view": {"algorithmic_bytes_per_launch": (8.0 * nf + 52.0) * ncell,
                             "achieved_gbs": (8.0 * nf + 52.0) * ncell / op_launch_s / 1e9 if op_launch_s else None,
                             "peak_gbs": peak, "peak_source": peak_kind}}
    # the formal-solver sweep: HBM roofline, chi and Snu read once per ray point frequency
    bytes_launch = 8.0 * ncell * nf
    achieved = bytes_launch / (sv_tot / sv_n / 1e3) / 1e9 if sv_n else None
    roofline_sweep = {"kernel": "k_quad_rot_column2 (rotate_array + long_char_quadratic, all slabs, one ray)",
                      "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                      "frac": achieved / peak if achieved else None,
                      "traffic": NCU_SWEEP_DRAM_BYTES_PER_CELL_FREQ * ncell * nf, "peak_source": peak_kind,
                      "algorithmic_bytes_per_launch": bytes_launch}
    # the same launch against instruction issue, the bound its arithmetic sets: the
    # quadratic step's real(4) operations are the reference's
    sv_inst = NCU_SWEEP_WARP_INST_PER_CELL_FREQ * ncell * nf
    sv_launch_s = sv_tot / sv_n / 1e3 if sv_n else None
    roofline_sweep["issue_view"] = {"warp_instructions_per_launch": sv_inst,
                                    "achieved": sv_inst / sv_launch_s / 1e9 if sv_launch_s else None,
                                    "peak": issue_peak, "unit": "G warp-instructions/s",
                                    "frac": sv_inst / sv_launch_s / 1e9 / issue_peak if sv_launch_s else None,
                                    "hbm_frac_at_full_issue": 8.0 * ncell * nf / (sv_inst / issue_peak) / peak}
    stages = {"opacity_ms_per_step": op_ms, "opacity_launches": op_n, "solve_ms_per_step": sv_ms,
              "solve_launches": sv_n, "reduce_ms_per_step": rd_ms, "windows": a.steps,
              "kernel_ms_per_step": op_ms + sv_ms + rd_ms,
              "outside_kernels_ms_per_step": ms / a.steps - (op_ms + sv_ms + rd_ms),
              "solve_gpt_per_s": work_per_step / (sv_ms / 1e3) / 1e9 if sv_ms else None}

    # end to end through the C ABI with pinned host buffers (copies inside the timed region)
    def pin(x):
        t = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
        return t.numpy()

    hatm = {k: (pin(v) if isinstance(v, np.ndarray) else v) for k, v in atm.items()}
    hatm["species"] = [{k: pin(v) for k, v in sp.items()} for sp in atm["species"]]
    hwin = [tuple(pin(x) for x in _window(llam_all, nu_all, nf, w)) for w in wins]
    h2d = sum(v.nbytes for k, v in hatm.items() if isinstance(v, np.ndarray))
    h2d += sum(v.nbytes for sp in hatm["species"] for v in sp.values()) + 2 * nf * 8
    d2h = (nray + 1) * nf * 4
    m.lte_synthesis(hatm, hwin[0][0], hwin[0][1], vec, wmu)
    e2e_steps = max(1, min(a.steps, 4))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        nu_h, llam_h = hwin[a.warmup + i % a.steps]
        ie, flux, _ = m.lte_synthesis(hatm, nu_h, llam_h, vec, wmu)
        float(flux[0])
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e = {"value": ws * work_per_step / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_s * 1e3}

    # the plain FP64 path on the same window (FP64 end to end: line opacity, QLG-bot,
    # transfer units, rotate_array and the quadratic solver), and the FP32 error
    # against it for each output
    fp64 = None
    if not a.no_fp64:
        nu_d, llam_d = dwin[a.warmup]
        ie32, f32, it32 = m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True, return_itop=True)
        torch.cuda.synchronize()
        # the FP32 pass timed on this same window, the ratio's numerator
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True)
        e1.record(stream)
        torch.cuda.synchronize()
        t32 = e0.elapsed_time(e1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ie64, f64, it64 = m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True, fp64=True, return_itop=True)
        e1.record(stream)
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1)

        def rel(x, y):
            r = (torch.abs(x.double() - y.double()) / torch.clamp(torch.abs(y.double()), min=1e-300)).flatten()
            med = float(r[:: max(1, r.numel() // 1000000)].median().item())
            return {"max": float(r.max().item()), "median": med}

        errors = {"flux": rel(f32, f64), "ie": rel(ie32, ie64), "I_top": rel(it32, it64)}
        del it32, it64
        c32, s32 = m.lte_transfer_units(datm, nu_d, llam_d, vec[6], device=True)
        c64, s64 = m.lte_transfer_units(datm, nu_d, llam_d, vec[6], device=True, fp64=True)
        torch.cuda.synchronize()
        errors["chi"] = rel(c32, c64)
        errors["S"] = rel(s32, s64)
        del c32, s32, c64, s64
        torch.cuda.empty_cache()
        m.profile_enable(True)
        m.lte_synthesis(datm, nu_d, llam_d, vec, wmu, device=True, fp64=True)
        op64_ms, _ = m.profile_read(m.STAGE_OPACITY)
        sv64_ms, sv64_n = m.profile_read(m.STAGE_SOLVE)
        m.profile_enable(False)
        fp64 = {"value": work_per_step / (t64 / 1e3) / 1e9, "unit": UNIT, "ms_per_step": t64,
                "fp32_over_fp64": t64 / t32, "fp32_ms_same_window": t32,
                "window": int(wins[a.warmup]),
                "fp32_error_vs_fp64": errors,
                "error_note": "relative; chi and S of ray 7 (mu 0.45), I_top every column and ray, ie and flux of "
                              "the window; single points of chi/S/I_top can differ by a QLG table node (FP32 and "
                              "FP64 snap a point to neighbouring nodes)",
                "opacity_ms_per_step": op64_ms, "solve_ms_per_step": sv64_ms, "solve_launches": sv64_n,
                "opacity_fp32_over_fp64": op64_ms / op1_ms if op1_ms else None,
                "solve_fp32_over_fp64": sv64_ms / sv1_ms if sv1_ms else None,
                "path": "FP64 end to end: line opacity and QLG-bot (fp64 tables, exp, log), transfer units, "
                        "rotate_array and long_char_quadratic, one launch per ray and slab"}

    nlte = batched = optab = continuum = None
    if rank == 0 and not a.no_ali:
        nlte = _nlte_ali()
        batched = _nlte_batched()
    if rank == 0 and not a.no_optab:
        optab = _optab()
        continuum = _continuum(sm_mhz=clocks.get("sm_mhz"))

    c0 = c4 = None
    if rank == 0 and not a.no_c0:
        c0 = _c0(m, a)
    if rank == 0 and not a.no_c4:
        c4 = _c4(m)
        m.set_stream(stream.cuda_stream or 1)

    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        # the same block sampler as the reference arm, the first timed window
        ref = CpuReference(atm, vec, wmu, ncols=REF_NCOLS)
        nu, llam = _window(llam_all, nu_all, nf, wins[a.warmup])
        ref.step(nu, llam)
        t0 = time.perf_counter()
        ref.step(nu, llam)
        dt = time.perf_counter() - t0
        ref.close()
        cpu = {"value": ref.work * nf / dt / 1e9, "unit": UNIT, "cores": ref.cores, "kind": "port",
               "sample": ref.describe(nf, dt)}

    if ws > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded grey cube, random line list)",
            "config": {**_workload(nf, a.cube), "windows_timed_rank0": wins[a.warmup:]},
            "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "roofline_sweep": roofline_sweep,
            "cpu_baseline": cpu, "clocks": clocks, "stages": stages, "fp64_plain": fp64, "c0_1d": c0, "c4_adjoint": c4,
            "nlte_ali": nlte, "nlte_batched": batched, "optab": optab, "continuum": continuum}
    print(json.dumps(line), flush=True)


def _c2_full(iters=30):
    """The 3D NLTE configuration in full: the 120^3 cube, the 20-level atom with its 80
    transitions in 8 windows of 250 frequencies (2000 in all), 26 directions (Lobatto
    4x4 and its mirror), short_char with split rates, lineq_no_pivot, Ng on its
    automatic gate; up to 30 ALI iterations to convlim 1e-3.  Returns the convergence
    history (maxerr and Ng per iteration) and the sweep and update times (CUDA events
    on torch's stream)."""
    import torch

    from dispatch_b200 import ali, synth
    cube, atom, _, vec, wts = ali.cube_problem("c2")
    nrad = len(atom["ti"])
    wins = [synth.atom_window(atom, seed=2, transitions=list(range(k, nrad, 8))) for k in range(8)]
    A = ali.AliCube(cube, atom, wins, vec, wts, params=ali.AliParams(convlim=1e-3))
    cur = torch.cuda.current_stream()
    hist, sw, up = [], [], []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    A.sweep()
    e1.record(cur)
    torch.cuda.synchronize()
    sw.append(e0.elapsed_time(e1))
    from dispatch_b200.stateq import NonFiniteSolution
    failure = None
    while A.iter < iters and not A.converged:
        A.iter += 1
        e0.record(cur)
        try:
            rec = A.update()
        except NonFiniteSolution as e:
            # update_populations stops the run here, as the reference's error stop does
            failure = {"iter": A.iter, "error": str(e).splitlines()[0]}
            break
        e1.record(cur)
        torch.cuda.synchronize()
        up.append(e0.elapsed_time(e1))
        ng = rec.get("ng") or {}
        hist.append({"iter": rec["iter"], "maxerr": rec["maxerr"], "ng_applied": bool(ng.get("applied", False))})
        if not A.converged and A.iter < iters:
            e0.record(cur)
            A.sweep()
            e1.record(cur)
            torch.cuda.synchronize()
            sw.append(e0.elapsed_time(e1))
    pts = A.points()
    out = {"workload": "c2 3D NLTE: 120^3 cube, 20-level atom, 80 transitions in 8 windows (2000 frequencies), "
                       "26 directions, short_char with split rates, lineq_no_pivot, Ng automatic, convlim 1e-3, "
                       f"at most {iters} iterations", "unit": UNIT,
           "iterations": A.iter, "converged": bool(A.converged), "history": hist, "stopped": failure,
           "sweep_ms_median": float(np.median(sw)), "update_ms_median": float(np.median(up)) if up else None,
           "total_s": (sum(sw) + sum(up)) / 1e3, "ray_pt_nu_per_sweep": pts,
           "value": pts / (float(np.median(sw)) / 1e3) / 1e9,
           "data": "synthetic (seeded grey cube, seeded model atom)"}
    del A
    torch.cuda.empty_cache()
    return out


def run_case_ali(a):
    """ALI iterations of a seeded problem, one line per iteration (the sweep and
    update times from CUDA events on torch's stream)."""
    import torch

    import dispatch_b200 as m
    from dispatch_b200 import ali
    m.init(0)
    t0 = time.time()
    if a.case == "ali-window":
        nrad = a.nline + a.nbound
        cube, atom, win, vec, wts = ali.cube_problem("small", nx=a.n, ny=a.n, nz=a.n, nbound=a.nbound,
                                                     nline=a.nline, ntheta=4, nphi=4,
                                                     transitions=list(range(0, nrad, a.every)))
        A = ali.AliWindow(cube, atom, win, vec, wts, params=ali.AliParams(convlim=1e-9))
    else:
        cols, atom, wins, mu, wmu = ali.column_problem(ncol=a.ncol, depth=(60, 256), nz=256, nxy=64,
                                                       nbound=a.nbound, nline=a.nline, nwin=a.nwin)
        A = ali.AliColumns(cols, atom, wins, mu, wmu, params=ali.AliParams(convlim=1e-9), use_graph=not a.no_graph,
                           fused=not a.per_point)
        print(f"plan shape {A.shape}", flush=True)
    torch.cuda.synchronize()
    print(f"setup {time.time() - t0:.1f} s, {A.ncell} cells, {A.points():.3e} ray-point-frequencies per sweep",
          flush=True)
    cur = torch.cuda.current_stream()
    A.sweep()
    for _ in range(a.iters):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(cur)
        A.iter += 1
        rec = A.update()
        e[1].record(cur)
        A.sweep()
        e[2].record(cur)
        torch.cuda.synchronize()
        sw = e[1].elapsed_time(e[2])
        print(f"iter {A.iter}: update {e[0].elapsed_time(e[1]):.1f} ms, sweep {sw:.1f} ms "
              f"({A.points() / sw / 1e6:.2f} Gpt/s), maxerr {rec['maxerr']:.3e}", flush=True)


def run_case_optab(a):
    """The two table samplers on a seeded n^3 cube, one window of --nf frequencies
    at R = 1e5: best of --iters, CUDA events on torch's stream."""
    import torch

    import dispatch_b200 as m
    from dispatch_b200 import synth
    from dispatch_b200.optab import SampleOptab
    m.init(0)
    c = synth.optab_cells(7, a.n, a.n, a.n)
    ncell = c["temp"].size
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    T, N, X, V = dev(c["temp"]), dev(c["ne"]), dev(c["chi500"]), dev(c["vproj"])
    back = torch.empty((ncell, a.nf), dtype=torch.float32, device="cuda")
    scat, xh, eh, cs = (torch.zeros_like(back) for _ in range(4))
    lam_q, bg, ll = synth.window_tables(8, c["temp"], c["ne"], c["vproj"], nf=a.nf)
    q = dev(lam_q)
    for name, tab in (("sample", bg), ("ll", ll)):
        if a.only and a.only != name:
            continue
        t = SampleOptab.from_dict(tab)
        ts = []
        for _ in range(a.iters):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if name == "sample":
                t.interpolate(T, N, X, q, back, scat)
            else:
                t.interpolate_ll(T, N, X, xh, eh, q, V, cs)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        print(f"{name}: {ncell} cells x {a.nf} frequencies, table {t.nnu} x {t.ntemp} x {t.nne}: "
              f"{min(ts):.3f} ms, {ncell * a.nf / min(ts) / 1e6:.2f} Gpt*nu/s", flush=True)
        t.close()


def main():
    a = _args()
    if a.case == "c2":
        import dispatch_b200 as m
        m.init(0)
        print(json.dumps(_c2_full(a.iters if a.iters != 2 else 30)), flush=True)
    elif a.case == "continuum":
        import dispatch_b200 as m
        m.init(0)
        print(json.dumps(_continuum(n=a.n)), flush=True)
    elif a.case == "c0":
        import dispatch_b200 as m
        m.init(0)
        print(json.dumps(_c0(m, a)), flush=True)
    elif a.case == "batched":
        import dispatch_b200 as m
        m.init(0)
        print(json.dumps(_nlte_batched()), flush=True)
    elif a.case in ("ali-window", "ali-columns"):
        run_case_ali(a)
    elif a.case == "optab":
        run_case_optab(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()

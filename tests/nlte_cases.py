"""Seeded inputs of the model-atom opacity and rate tests: the 21-level atom on
its 2000-point window and a few hundred cells of the small cube, with a
synthetic radiation field where a test does not form one from the opacities."""
import numpy as np

from dispatch_b200 import synth

_EE, _BK, _HH = synth.EE, synth.BK, synth.HH


def case(ncell=300, seed=11, sums_every=0, cut_x=70.0):
    atom, inp = synth.se_config("small", ncell=ncell)
    sums = None
    if sums_every:
        sums = (np.arange(atom["nline"]) % sums_every == 0).astype(np.uint8)
    win = synth.atom_window(atom, sums=sums)
    win["cut_x"] = cut_x
    rng = np.random.default_rng(seed)
    nf = win["nf"]
    temp = inp["temp"]
    cells = {
        "b": inp["b"], "nstar": inp["nstar"], "pop_ratio": np.ones(ncell), "e_kT": inp["e_kT"],
        "inv_df": (1.8e5 * (1 + 0.1 * rng.standard_normal(ncell))).astype(np.float32),
        "vproj": (1e-5 * rng.standard_normal(ncell)).astype(np.float32),
        "ne": inp["ne"].astype(np.float32), "tothi": (1e4 * inp["ne"]).astype(np.float32),
        "vbar2": (1e10 * (1 + rng.random(ncell))).astype(np.float32),
        "stark_pe": (inp["ne"] * temp ** (1 / 6)).astype(np.float32),
        "unsold": ((1e10 * (1 + rng.random(ncell))) ** 0.3 * 1e4 * inp["ne"]).astype(np.float32),
    }
    hnu_kt = (_HH * win["nu"])[None, :] / (_BK * temp[:, None])
    beta = np.maximum(np.exp(-hnu_kt), np.finfo(np.float32).tiny).astype(np.float32)
    Bnu = (beta / (1 - beta)).astype(np.float32)
    field = {
        "beta": beta, "Bnu": Bnu,
        "xhat": (1e-8 * (1 + rng.random((ncell, nf)))).astype(np.float32),
        "ehat": (1e-8 * Bnu / beta * (1 + 0.2 * rng.random((ncell, nf)))).astype(np.float32),
        "inu": (Bnu * (0.3 + rng.random((ncell, nf)))).astype(np.float32),
        "psi": rng.random((ncell, nf)).astype(np.float32),
        "escape": rng.random((ncell, nf)).astype(np.float32),
    }
    field["irem"] = (field["inu"] * (0.2 + 0.5 * rng.random((ncell, nf)))).astype(np.float32)
    return atom, inp, win, cells, field

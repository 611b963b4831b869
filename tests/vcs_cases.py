"""Synthetic VCS table files in the format hvcs_mod.f90's read_vcs_grid reads: a
header of the log10 axes (delta-lambda from -2 in steps of 0.1, ne from 10 in
steps of 0.5, N(HI) from 12 in steps of 0.5, log T from log10(2500) in steps of
log10(2)), then per line "nlow nup nhhnr" and log10 profiles on 44 x nhhnr x 4 x 13
nodes.  The profiles are Lorentzian-like Stark shapes whose width grows with ne,
T and N(HI), smooth enough for the interpolations and with a power-law wing.
The real tables (Lemke 1997, Stehle & Hutcheon 1999) belong to the reference's
data; these stand in for them wherever the reference is not at hand."""
import numpy as np

SERIES = {1: [(2, 3, 13), (2, 4, 1), (2, 5, 13), (2, 12, 1), (2, 18, 1)],
          2: [(3, 4, 1), (3, 7, 1)],
          3: [(4, 7, 1), (4, 10, 1)]}


def write(path, series, seed=0):
    rng = np.random.default_rng(seed + series)
    dw = -2.0 + 0.1 * np.arange(44)
    lgt = np.log10(2500.0) + np.log10(2.0) * np.arange(4)
    lne = 10.0 + 0.5 * np.arange(13)
    lnh = 12.0 + 0.5 * np.arange(13)
    out = ["  -2.00    0.10   10.00    0.50   12.00    0.50   3.3979399   0.3010300"]
    for n, m, nn in SERIES[series]:
        out.append(f"{n:5d}{m:5d}{nn:5d}")
        vals = []
        a = rng.uniform(0.8, 1.2)
        for l in range(13):
            for kk in range(4):
                for j in range(nn):
                    w = a * 1e-3 * (m - n) ** 2 * 10 ** ((lne[l] - 12.0) * 0.66) * 10 ** ((lgt[kk] - 3.7) * 0.1)
                    w *= 1.0 + 0.05 * j
                    x = 10.0 ** dw
                    prof = w / np.pi / (x * x + w * w) * (1.0 + 0.3 * np.exp(-x / (3 * w)))
                    vals.append(np.log10(prof))
        v = np.concatenate(vals)
        for i in range(0, v.size, 11):
            out.append(" ".join(f"{x:8.4f}" for x in v[i:i + 11]))
    open(path, "w").write("\n".join(out) + "\n")


def write_all(folder, seed=0):
    import os
    paths = {}
    for s in (1, 2, 3):
        p = os.path.join(folder, f"synthetic_vcs_{s}.txt")
        write(p, s, seed)
        paths[s] = p
    return paths

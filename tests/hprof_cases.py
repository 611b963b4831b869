"""Seeded cells and hydrogen lines for the hydrogen profile tests: temperatures,
electron and neutral hydrogen densities spanning photospheres and chromospheres,
the derived Doppler width, Holtsmark field F0 = 1.25e-9 ne^(2/3) (HLINOP's
normal field strength), mean relative speed with H and the helium term."""
import numpy as np

CC = 2.99792458e10
LINES = [(1, 2, 1215.668), (1, 3, 1025.722), (2, 3, 6564.61), (2, 4, 4862.68), (2, 5, 4341.68),
         (2, 12, 3751.2), (2, 18, 3692.6), (3, 4, 18756.1), (3, 7, 10052.1), (4, 7, 21661.2), (5, 9, 38880.0)]


def cells(seed=1, n=257, ne_range=(9.0, 16.0)):
    rng = np.random.default_rng(seed)
    T = rng.uniform(3500.0, 12000.0, n)
    ne = 10.0 ** rng.uniform(*ne_range, n)
    nH = 10.0 ** rng.uniform(12.0, 17.0, n)
    mh, bk = 1.6726e-24, 1.380662e-16
    vth = np.sqrt(2 * bk * T / mh + (1e5 * rng.uniform(0.5, 2.0, n)) ** 2)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    return {"temp": f32(T), "ne": f32(ne), "tothi": f32(nH), "fo": f32(1.25e-9 * ne ** (2.0 / 3.0)),
            "vbar2h": f32(8 * bk * T / np.pi * (1 / mh + 1 / mh)), "t3nhe": f32((T / 1e4) ** 0.3 * 0.085 * nH),
            "inv_df": f32(CC / vth), "vproj": f32(rng.normal(0.0, 1e-5, n)),
            "ni": f32(10.0 ** rng.uniform(2.0, 8.0, n))}


def nu0(lam_aa):
    return CC * 1e8 / lam_aa


def grid(lam_aa, half_aa, nf):
    """A frequency grid uniform in wavelength over lam +- half, ascending in nu."""
    lam = np.linspace(lam_aa + half_aa, lam_aa - half_aa, nf)
    return CC * 1e8 / lam

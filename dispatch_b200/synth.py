"""Seeded synthetic atmospheres, line lists and frequency grids of the
benchmark configurations (stand-ins for real model atmospheres and line lists).

Grey atmosphere T^4 = 3/4 Teff^4 (tau + 2/3), Teff = 5800 K, log g = 4.4, a grey
continuum kappa500 = 0.2 cm^2/g of pure absorption, hydrostatic equilibrium with
mean molecular weight 1.26, n_H = rho/(1.4 m_H), n_e = 1e-4 n_H.  One line
absorber per species (mass 56 u, A = 7.50, U = 25, vmic = 1 km/s by default).
Random numbers: numpy PCG64 (default_rng(seed)).  3D cubes: a Gaussian random
temperature field (periodic, correlation exp(-r^2/2l^2)) on the grey model,
vertical velocities, density re-integrated hydrostatically per column.

The per-cell quantities the line kernel takes are formed exactly as
add_particle_opacity forms them (HOP/linelist_mod.f90:1000-1047,
HOP/ion_mod.f90:198-225).
"""
from __future__ import annotations

import math

import numpy as np

# const_mod.f90:38-73
EE = 1.602189e-12
HH = 6.626176e-27
CC = 2.99792458e10
EM = 9.109534e-28
UU = 1.6605655e-24
BK = 1.380662e-16
ECH = 4.80325e-10
MH = 1.6726e-24
PI = 3.14159265359
HZ_TO_AA = CC / 1e-8
F_CONV = 8.0 * PI**2 * ECH**2 / EM / CC**3      # bbtrans_mod.f90:47
C2_2H = CC**2 / 2.0 / HH
H_4PI = HH * (1.0 / (4.0 * PI))
BIJ_CONST = C2_2H * F_CONV * H_4PI               # linelist_mod.f90:53

TEFF, LOGG, KAPPA500, MU_MOL = 5800.0, 4.4, 0.2, 1.26


def grey_temperature(tau):
    return (0.75 * TEFF**4 * (tau + 2.0 / 3.0)) ** 0.25


def grey_model(log_tau):
    """T, P, rho, n_H, n_e of the grey model at log10 tau500 (any shape)."""
    tau = 10.0 ** np.asarray(log_tau, np.float64)
    g = 10.0**LOGG
    T = grey_temperature(tau)
    P = g * tau / KAPPA500
    rho = P * MU_MOL * MH / (BK * T)
    nH = rho / (1.4 * MH)
    return T, P, rho, nH, 1e-4 * nH


def random_linelist(rng, n, lam0, lam1, loggf=(-3.0, 0.0), elow=(0.0, 5.0), adamp=(1e-3, 1e-1)):
    """Lines uniform in [lam0, lam1] AA, sorted; returns raw parameters."""
    lam = np.sort(rng.uniform(lam0, lam1, n))
    return {"lam": lam, "loggf": rng.uniform(*loggf, n), "elow": rng.uniform(*elow, n),
            "adamp": 10.0 ** rng.uniform(math.log10(adamp[0]), math.log10(adamp[1]), n)}


def inverse_doppler_factor(temp, awgt, vmic_kms):
    """ion_mod.f90:198-211, in real(4)."""
    const = np.float32(2.0 * BK / UU)
    temp = np.asarray(temp, np.float32)
    dop = (const * temp) / np.float32(awgt)
    if vmic_kms > 0:
        dop = dop + np.float32((vmic_kms * 1e5) ** 2)
    return (np.float32(CC) / np.sqrt(dop)).astype(np.float32)


def compute_vbar2(temp, awgt):
    """ion_mod.f90:214-225, in real(4)."""
    const = np.float32(8.0 * BK / (PI * UU))
    inv_mh = np.float32(UU / MH)
    temp = np.asarray(temp, np.float32)
    return ((const * temp) * (inv_mh + np.float32(1.0) / np.float32(awgt))).astype(np.float32)


def species_arrays(raw, temp, n_x, awgt=56.0, part=25.0, vmic_kms=1.0):
    """Line-list SoA and per-cell fields of one species (one isotope).

    gpref = loggf ln10 + ln(bij_const/nu0) (line_types_mod.f90:30-35); the damping
    drawn in Doppler widths is folded in as grad = a/idf at Teff, with no van der
    Waals or Stark term (gw1 = gstk = 0)."""
    lam = raw["lam"]
    nu0 = HZ_TO_AA / lam
    idf_ref = float(inverse_doppler_factor(np.float32(TEFF), awgt, vmic_kms))
    n = lam.size
    ll = {
        "llam0": np.log(lam).astype(np.float64),
        "lower_ev": raw["elow"].astype(np.float32),
        "gpref": (raw["loggf"] * math.log(10.0) + np.log(BIJ_CONST / nu0)).astype(np.float32),
        "grad": (raw["adamp"] / idf_ref).astype(np.float32),
        "gw1": np.zeros(n, np.float32),
        "gw2": np.zeros(n, np.float32),
        "gstk": np.zeros(n, np.float32),
        "unsold": np.zeros(n, np.uint8),
    }
    idf = inverse_doppler_factor(temp, awgt, vmic_kms)
    vb2 = compute_vbar2(temp, awgt)
    lnb = (np.log(np.maximum(np.asarray(n_x, np.float64), np.finfo(np.float64).tiny)).astype(np.float32)
           - np.float32(math.log(part)) + np.log(idf).astype(np.float32))
    ll.update({"inv_df": idf, "vbar2": vb2, "lnbase": lnb.astype(np.float32)})
    return ll


def cell_fields(temp, nH, ne):
    """e_kT, ne, tothi, stark_pe per cell (composition_mod.f90:1719-1724)."""
    temp = np.asarray(temp, np.float32)
    return {"e_kT": (np.float32(EE / BK) / temp).astype(np.float32),
            "ne": np.asarray(ne, np.float32),
            "tothi": np.asarray(nH, np.float32),
            "stark_pe": (np.asarray(ne, np.float32) * temp ** np.float32(1.0 / 6.0)).astype(np.float32)}


def frequency_grid(lam0, lam1, nf):
    """Uniform in ln(lambda): returns (llam, nu) ascending in llam."""
    llam = np.linspace(math.log(lam0), math.log(lam1), nf)
    return llam, HZ_TO_AA / np.exp(llam)


def gaussian_field(rng, shape, ell, sigma):
    """Periodic Gaussian random field with correlation exp(-r^2/2 ell^2), scaled to sigma."""
    white = rng.standard_normal(shape)
    if sigma == 0.0:
        return np.zeros(shape)
    k = [np.fft.fftfreq(n) * 2 * np.pi for n in shape]
    kk = np.zeros(shape)
    for i, ki in enumerate(k):
        s = [1] * len(shape)
        s[i] = -1
        kk = kk + ki.reshape(s) ** 2
    sk = ell / math.sqrt(2.0)
    filt = np.exp(-0.5 * kk * sk**2)
    f = np.real(np.fft.ifftn(np.fft.fftn(white) * filt))
    f -= f.mean()
    return f * (sigma / f.std())


def cube_atmosphere(seed, nx, ny, nz, sigma_t=300.0, ell=8.0, sigma_vz_kms=2.0, log_tau=(-6.0, 2.0), aspect=2.0):
    """3D cube, z index 0 = bottom (deepest).  Returns dict of (nz, ny, nx) arrays
    plus the cell size [cm]; the horizontal cell size is aspect times the vertical."""
    rng = np.random.default_rng(seed)
    # mean model on a fine tau grid -> geometric depth
    lt = np.linspace(log_tau[1], log_tau[0], 4001)
    T, P, rho, nH, _ = grey_model(lt)
    tau = 10.0**lt
    dz = np.concatenate([[0.0], -np.diff(tau) / (KAPPA500 * 0.5 * (rho[1:] + rho[:-1]))])
    height = np.cumsum(dz)                      # 0 at the bottom (tau = 100), increasing upwards
    zc = np.linspace(0.0, height[-1], nz + 1)
    zc = 0.5 * (zc[1:] + zc[:-1])
    ds_z = zc[1] - zc[0]
    ltz = np.interp(zc, height, lt)
    T0 = grey_temperature(10.0**ltz)
    dT = gaussian_field(rng, (nz, ny, nx), ell, sigma_t)
    temp = np.maximum(T0[:, None, None] + dT, 2500.0)
    vz = gaussian_field(rng, (nz, ny, nx), ell, sigma_vz_kms) * 1e5
    # hydrostatic per column from the top down: dP/dz = -rho g, rho = P mu m_H/(kT)
    g = 10.0**LOGG
    P = np.empty_like(temp)
    _, Ptop, _, _, _ = grey_model(ltz[-1])
    P[-1] = Ptop
    for k in range(nz - 2, -1, -1):
        Tm = 0.5 * (temp[k] + temp[k + 1])
        P[k] = P[k + 1] * np.exp(g * MU_MOL * MH / (BK * Tm) * ds_z)
    rho = P * MU_MOL * MH / (BK * temp)
    nH = rho / (1.4 * MH)
    ds_xy = ds_z * aspect
    return {"temp": temp.astype(np.float32), "rho": rho, "nH": nH, "ne": 1e-4 * nH,
            "chi_c": (KAPPA500 * rho).astype(np.float32), "vz": (vz / CC).astype(np.float32),
            "ds_cm": (ds_xy, ds_xy, ds_z)}


def column_set(seed=3, ncol=4096, depth=(60, 256), nz=256, nxy=64, variants=(0.0,), sigma_t=300.0):
    """Columns of uneven depth drawn from a seeded cube (the batched 1.5D
    configuration): the cube_atmosphere of nxy^2 columns and nz planes, ncol of its
    columns, each cut to its top d cells with d uniform in depth (inclusive).  The
    columns are packed back to back, bottom to top, once per abundance variant
    (a dex offset each).  Returns the per-cell fields (temp, ne, nH, chi_c, vz,
    abund_dex), col_off (ncol*len(variants)+1), dz per column [cm] and the column
    of the cube each packed column came from."""
    c = cube_atmosphere(seed, nxy, nxy, nz, sigma_t=sigma_t)
    rng = np.random.default_rng(seed + 6000)
    pick = rng.choice(nxy * nxy, size=ncol, replace=ncol > nxy * nxy)
    d = rng.integers(depth[0], depth[1] + 1, size=ncol)
    d = np.minimum(d, nz)
    fields = {k: [] for k in ("temp", "ne", "nH", "chi_c", "vz", "abund_dex")}
    off = [0]
    src = []
    for v in variants:
        for j, (col, dj) in enumerate(zip(pick, d)):
            y, x = divmod(int(col), nxy)
            zs = slice(nz - int(dj), nz)
            for k in ("temp", "ne", "nH", "chi_c", "vz"):
                fields[k].append(np.asarray(c[k])[zs, y, x])
            fields["abund_dex"].append(np.full(int(dj), float(v)))
            off.append(off[-1] + int(dj))
            src.append(int(col))
    out = {k: np.concatenate(v) for k, v in fields.items()}
    out["temp"] = out["temp"].astype(np.float32)
    out["chi_c"] = out["chi_c"].astype(np.float32)
    out["vz"] = out["vz"].astype(np.float32)
    out["col_off"] = np.asarray(off, np.int32)
    out["dz"] = np.full(len(src), float(c["ds_cm"][2]))
    out["source_column"] = np.asarray(src, np.int64)
    return out


def column_1d(ndep=80, log_tau=(-6.0, 2.0)):
    """The 1D grey model on log tau uniform, z index 0 = bottom."""
    lt = np.linspace(log_tau[1], log_tau[0], ndep)
    T, P, rho, nH, ne = grey_model(lt)
    tau = 10.0**lt
    dz = -np.diff(tau) / (KAPPA500 * 0.5 * (rho[1:] + rho[:-1]))
    return {"temp": T.astype(np.float32), "rho": rho, "nH": nH, "ne": ne,
            "chi_c": (KAPPA500 * rho).astype(np.float32), "dz": dz}


def lobatto_rays(ntheta=4, nphi=4, jnu_weights=False):
    """set_lobatto_quadratures + nphi_copies (SRC/ray_mod.f90:224-262, 392-490):
    mu = 1 once, every other mu with nphi azimuths.  The table is the reference's
    default-real literals, so mu and the weights are float32 values.  Flux
    weights wmu/nphi times mu; with jnu_weights the set mirrored to the
    downward hemisphere (vec -> -vec) and the weights halved."""
    tab = {4: ([1.0, 0.87174015, 0.59170018, 0.20929922], [0.03571428, 0.21070422, 0.34112270, 0.41245880]),
           3: ([1.0, 0.76505532, 0.28523152], [0.06666667, 0.37847496, 0.55485838]),
           2: ([1.0, 0.44721360], [0.16666667, 0.83333333]),
           1: ([1.0], [1.0])}
    mu, wmu = tab[ntheta]
    return _nphi_copies(nphi, _f32(mu), _f32(wmu), jnu_weights=jnu_weights)


def gauss_rays(ntheta=5, nphi=1, jnu_weights=False):
    """set_gauss_quadratures: Gauss-Legendre mu on (0, 1), descending, rounded to
    float32 as the reference's default-real table is; then nphi_copies."""
    x, w = np.polynomial.legendre.leggauss(ntheta)
    mu = 0.5 * (x + 1.0)
    wmu = 0.5 * w
    order = np.argsort(-mu)
    return _nphi_copies(nphi, _f32(mu[order]), _f32(wmu[order]), jnu_weights=jnu_weights)


def radau_nodes(k: int):
    """radau%init (solvers/rt/radau_mod.f90): the k-point Gauss-Radau rule on
    [-1, 1] with the fixed node -1, mapped to mu = 1 - (x + 1)/2 on [0, 1] with
    weights w/2, in real(4) as the reference stores them; ascending in mu.  The
    free nodes are the roots of (P_{k-1} + P_k)/(1 + x) and their weights
    (1 - x)/(k P_{k-1}(x))^2 (the rule the reference tabulates for k <= 10)."""
    if not 1 <= k <= 10:
        raise ValueError("Radau quadrature: 1 <= ntheta <= 10")
    if k == 1:
        x, w = np.array([-1.0]), np.array([2.0])
    else:
        c = np.zeros(k + 1)
        c[k - 1] = c[k] = 1.0
        x = np.sort(np.real(np.polynomial.legendre.legroots(c)))
        x[0] = -1.0
        pk1 = np.polynomial.legendre.legval(x, np.eye(k)[k - 1])
        w = (1.0 - x) / (k * k * pk1 * pk1)
        w[0] = 2.0 / (k * k)
    # xi(i) = 1 - (c + d xn(k0(k+1)-i)): the table's nodes from the last down
    mu = (1.0 - (0.5 + 0.5 * x[::-1])).astype(np.float32)
    wmu = (0.5 * w[::-1]).astype(np.float32)
    return mu, wmu


def radau_rays(ntheta=2, nphi=1, jnu_weights=False):
    """set_radau_quadratures (SRC/ray_mod.f90:365-384): Radau mu including 1,
    descending, azimuths rotated by zrot = pi/4, then nphi_copies."""
    mu2, wmu2 = radau_nodes(ntheta)
    mu = mu2[::-1].astype(np.float64)
    wmu = wmu2[::-1].astype(np.float64)
    return _nphi_copies(nphi, mu, wmu, zrot=np.full(ntheta, PI / 4.0), jnu_weights=jnu_weights)


def _f32(v):
    return np.asarray(np.asarray(v, np.float32), np.float64)


def _nphi_copies(nphi, mu, wmu, zrot=None, jnu_weights=False, one_dimensional=False):
    """nphi_copies (SRC/ray_mod.f90:392-465)."""
    nphi = 1 if one_dimensional else nphi
    vec, wts = [], []
    for k, (m, w) in enumerate(zip(mu, wmu)):
        if m == 1.0:
            vec.append([0.0, 0.0, 1.0])
            wts.append(w)
            continue
        th = math.acos(m)
        xoff = 0.0 if zrot is None else float(zrot[k])
        for p in range(nphi):
            ph = 2.0 * PI / nphi * p + xoff
            v = [math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), m]
            v = [0.0 if abs(c) < 1e-3 else c for c in v]
            vec.append(v)
            wts.append(w / nphi)
    vec = np.array(vec, np.float64)
    wts = np.array(wts, np.float64)
    if jnu_weights:
        return np.concatenate([vec, -vec]), np.concatenate([wts, wts]) / 2.0
    return vec, wts * vec[:, 2]


def lte_config(kind: str, seed: int | None = None, nf: int | None = None, window: int = 0,
               cube=None, lines=None, size: int | None = None):
    """Inputs of one frequency window of a configuration, ready for
    m3d_lte_synthesis.

    kind: 'c0' (1D, 80 depths, 2000 lines in 5000-5100 AA, 20000 freq, 5 Gauss mu),
          'c1' (3D 240^3 in 10 slabs, 500 lines in 5000-5020 AA, 4000 freq, 13 rays),
          'mini' (a small 3D case for tests: 16x12x10, 2 slabs, 60 lines).
    size: an n^3 cube in place of the configuration's own (same lines, slabs, rays).
    nf: frequencies per window (the run's n_windows split); window: which one."""
    if kind == "c0":
        seed = 0 if seed is None else seed
        nxyz, nfree, lam = (1, 1, 80), 20000, (5000.0, 5100.0)
        nline, nslab = 2000, 1
    elif kind == "c1":
        seed = 1 if seed is None else seed
        nxyz, nfree, lam = (240, 240, 240), 4000, (5000.0, 5020.0)
        nline, nslab = 500, 10
    elif kind == "mini":
        seed = 7 if seed is None else seed
        nxyz, nfree, lam = (16, 12, 10), 400, (5000.0, 5004.0)
        nline, nslab = 60, 2
    else:
        raise ValueError(kind)
    if size is not None:
        nxyz = (size, size, size)
    nf = nfree if nf is None else nf
    rng = np.random.default_rng(seed + 1000)
    if lines is None:
        lines = random_linelist(rng, nline, *lam)
    nx, ny, nz = nxyz
    if cube is None:
        if kind == "c0":
            # the grey column on 80 planes uniform in height over log tau500 in [-6, 2]
            cube = cube_atmosphere(seed, 1, 1, nz, sigma_t=0.0, sigma_vz_kms=0.0, log_tau=(-6.0, 2.0))
        else:
            cube = cube_atmosphere(seed, nx, ny, nz)
    temp, rho, nH, ne, chi_c, vz = (cube[k] for k in ("temp", "rho", "nH", "ne", "chi_c", "vz"))
    ds_cm = cube["ds_cm"]
    n_x = 10.0 ** (7.5 - 12.0) * nH
    sp = species_arrays(lines, temp, n_x)
    cf = cell_fields(temp, nH, ne)
    llam_all, nu_all = frequency_grid(lam[0], lam[1], nfree)
    sl = slice(window * nf, (window + 1) * nf)
    ds_code = tuple(d / 1e8 for d in ds_cm)
    slab_nz = [nz // nslab] * nslab
    slab_nz[-1] += nz - sum(slab_nz)
    atm = {"nx": nx, "ny": ny, "nz": nz, "slab_nz": slab_nz, "ds_cm": ds_cm, "ds_code": ds_code,
           "pivot_z": nz * ds_code[2], "ray_offset": (0.0, 0.0),
           "temp": np.ascontiguousarray(temp, np.float32).ravel(),
           "chi_c": np.ascontiguousarray(chi_c, np.float32).ravel(),
           "vx": np.zeros(temp.size, np.float32), "vy": np.zeros(temp.size, np.float32),
           "vz": np.ascontiguousarray(vz, np.float32).ravel(),
           "species": [{k: (np.ascontiguousarray(v).ravel() if k in ("inv_df", "vbar2", "lnbase") else v)
                        for k, v in sp.items()}]}
    atm.update({k: np.ascontiguousarray(v, np.float32).ravel() for k, v in cf.items()})
    vec, wmu = gauss_rays(5) if kind == "c0" else lobatto_rays(4, 4)
    return atm, np.ascontiguousarray(nu_all[sl]), np.ascontiguousarray(llam_all[sl]), vec, wmu


# ---- the differentiable configuration: ten species ------------------------------------
# (element, atomic mass [u], abundance log eps with log eps(H) = 12): a fixed table of
# ten metals at roughly solar abundances, the species of the synthetic line list
C4_SPECIES = (("Fe", 55.845, 7.50), ("Ti", 47.867, 4.95), ("Cr", 51.996, 5.64), ("Ni", 58.693, 6.22),
              ("Ca", 40.078, 6.34), ("Mg", 24.305, 7.60), ("Si", 28.086, 7.51), ("Na", 22.990, 6.24),
              ("Mn", 54.938, 5.43), ("Co", 58.933, 4.99))


def lte_config_c4(seed: int = 4, size=None, nf: int = 32, window: int = 0, nline_per_species: int = 100,
                  nfree: int = 8000, lam=(6000.0, 6050.0), cube=None):
    """One window of the differentiable 3D LTE configuration: a 96x96x128 seeded cube
    (cube_atmosphere, 8 slabs of 16 planes), 100 lines per species of the ten in
    C4_SPECIES, uniform in 6000-6050 A, 8000 frequencies uniform in ln(lambda), 13
    Lobatto rays.  size = (nx, ny, nz) for a smaller cube.  Returns (atm, nu, llam,
    vec, wmu, raw): raw holds what a differentiable caller re-forms the per-cell fields
    from -- temp, nH, the species' masses, abundances and raw line parameters."""
    nx, ny, nz = (96, 96, 128) if size is None else size
    rng = np.random.default_rng(seed + 1000)
    if cube is None:
        cube = cube_atmosphere(seed, nx, ny, nz)
    temp, nH, ne, chi_c, vz = (cube[k] for k in ("temp", "nH", "ne", "chi_c", "vz"))
    species, raws = [], []
    for name, awgt, abund in C4_SPECIES:
        raw = random_linelist(rng, nline_per_species, *lam)
        n_x = 10.0 ** (abund - 12.0) * nH
        sp = species_arrays(raw, temp, n_x, awgt=awgt)
        species.append({k: (np.ascontiguousarray(v).ravel() if k in ("inv_df", "vbar2", "lnbase") else v)
                        for k, v in sp.items()})
        raws.append(raw)
    llam_all, nu_all = frequency_grid(lam[0], lam[1], nfree)
    sl = slice(window * nf, (window + 1) * nf)
    ds_cm = cube["ds_cm"]
    ds_code = tuple(d / 1e8 for d in ds_cm)
    nslab = max(1, nz // 16)
    slab_nz = [nz // nslab] * nslab
    slab_nz[-1] += nz - sum(slab_nz)
    atm = {"nx": nx, "ny": ny, "nz": nz, "slab_nz": slab_nz, "ds_cm": ds_cm, "ds_code": ds_code,
           "pivot_z": nz * ds_code[2], "ray_offset": (0.0, 0.0),
           "temp": np.ascontiguousarray(temp, np.float32).ravel(),
           "chi_c": np.ascontiguousarray(chi_c, np.float32).ravel(),
           "vx": np.zeros(temp.size, np.float32), "vy": np.zeros(temp.size, np.float32),
           "vz": np.ascontiguousarray(vz, np.float32).ravel(), "species": species}
    atm.update({k: np.ascontiguousarray(v, np.float32).ravel() for k, v in cell_fields(temp, nH, ne).items()})
    vec, wmu = lobatto_rays(4, 4)
    raw = {"temp": np.asarray(temp, np.float64).ravel(), "nH": np.asarray(nH, np.float64).ravel(),
           "awgt": [c[1] for c in C4_SPECIES], "abund": np.array([c[2] for c in C4_SPECIES]), "lines": raws,
           "llam_all": llam_all, "nu_all": nu_all}
    return atm, np.ascontiguousarray(nu_all[sl]), np.ascontiguousarray(llam_all[sl]), vec, wmu, raw


# ---- NLTE: a seeded model atom and the per-cell inputs of its SE update ---------------
RYDV = 13.605


def model_atom(seed: int = 2, nbound: int = 20, nline: int = 60, e_max: float = 7.0, e_ion: float = 7.9,
               logf=(-4.0, 0.0), h_recipes=None, awgt: float = 40.08, gencol: bool = False,
               min_line_ev: float = 0.0) -> dict:
    """A seeded model atom: nbound levels of the neutral (ground at 0 eV, the rest
    uniform in [0, e_max]) plus the ground level of the ion at e_ion; nline lines
    between distinct random bound pairs with log f uniform in logf; one continuum
    from every bound level to the ion; classic_col pairs as the reference fills
    them for an atom without collision data: van Regemorter for every bound pair
    (f of the pair's line, or 0) and Seaton for every continuum, whose alpha0 is
    the hydrogenic 7.91e-18 n_eff cm^2 for even levels and 0 (Kramers inside
    the collision recipe) for odd ones.  h_recipes = (h_excitation, h_ionisation,
    h_forbidden), e.g. ('drawin', 'drawin', 'takeda'), adds the hydrogen recipes
    of every pair (col_hkind): Takeda for a bound pair without a line, else
    Drawin.  awgt: the atom's weight [amu].  gencol adds tabulated collision
    records of every kind (model_gencol); classic_col then leaves out the recipes
    the records' data replaces, as the reference does.  min_line_ev: lines only
    between levels at least this far apart (0: any pair; the uniform level draw puts
    some pairs a few meV apart, whose lines sit in the far infrared and mm, where
    stimulated emission dominates and small population inversions make masers).
    Indices are 0-based."""
    rng = np.random.default_rng(seed + 2000)
    ev = np.concatenate([[0.0], np.sort(rng.uniform(0.0, e_max, nbound - 1)), [e_ion]])
    g = np.concatenate([rng.choice([1.0, 3.0, 5.0, 7.0, 9.0], nbound), [1.0]])
    ion = np.concatenate([np.ones(nbound, np.int32), [2]]).astype(np.int32)
    n = nbound + 1
    pairs = [(i, j) for i in range(nbound) for j in range(i + 1, nbound) if ev[j] - ev[i] >= min_line_ev]
    pick = np.sort(rng.choice(len(pairs), size=min(nline, len(pairs)), replace=False))
    lines = [pairs[p] for p in pick]
    f = 10.0 ** rng.uniform(*logf, len(lines))
    ti = [i for i, _ in lines] + list(range(nbound))
    tj = [j for _, j in lines] + [nbound] * nbound
    lam_aa = np.array([HH * CC / ((ev[j] - ev[i]) * EE) * 1e8 for i, j in lines])
    # A_ji = 6.670e15 g_i/g_j f / lambda[AA]^2
    aji = np.concatenate([6.670e15 * g[[i for i, _ in lines]] / g[[j for _, j in lines]] * f / lam_aa**2,
                          np.zeros(nbound)])
    fpair = {p: fv for p, fv in zip(lines, f)}
    col_i, col_j, col_kind, col_fac = [], [], [], []
    for i in range(nbound):
        for j in range(i + 1, n):
            if ion[j] > ion[i]:
                col_i.append(i)
                col_j.append(j)
                col_kind.append(2)
                col_fac.append(7.91e-18 * math.sqrt(RYDV / (e_ion - ev[i])) if i % 2 == 0 else 0.0)
            else:
                col_i.append(i)
                col_j.append(j)
                col_kind.append(1)
                col_fac.append(fpair.get((i, j), 0.0))
    gc, hkind = None, None
    if gencol:
        from .stateq import classic_pairs
        gc, ecol, hcol = model_gencol(n, nbound, seed)
        cdata = np.zeros((n, n), np.float32)
        cdata[col_i, col_j] = col_fac
        cp = classic_pairs(ion, np.where(ion == 1, nbound, -1), cdata, ecol=ecol, hcol=hcol,
                           **dict(zip(("h_excitation", "h_ionisation", "h_forbidden"), h_recipes or ("", "", ""))))
        col_i, col_j, col_kind, col_fac = cp["col_i"], cp["col_j"], cp["col_kind"], cp["col_fac"]
        hkind = cp["col_hkind"]
    else:
        hkind = _hydrogen_kinds(ion, col_i, col_j, col_fac, h_recipes)
    return {"nlevel": n, "g": g, "ev": ev, "ion": ion,
            "ti": np.array(ti, np.int32), "tj": np.array(tj, np.int32), "nline": len(lines),
            "Aji": aji, "active": None, "line_f": f,
            "col_i": np.array(col_i, np.int32), "col_j": np.array(col_j, np.int32),
            "col_kind": np.array(col_kind, np.int32), "col_fac": np.array(col_fac, np.float32),
            "fmin": float(np.float32(1e-6)), "cbbesc": 1.0, "cbfesc": 1.0, "colscale": 1.0,
            "upsilon_floor": 0.0, "cut_x": 70.0, "bf_cut_rate": 1.0, "awgt": float(awgt),
            "col_hkind": hkind, "gencol": gc}


def model_gencol(n: int, nbound: int, seed: int = 2, ntemp: int = 9):
    """Tabulated collision records for model_atom's levels (n = nbound + 1, the last
    the ion): every kind of record, two records on one level pair, one with its
    levels reversed, tables with a flat stretch and a turning point, on ntemp nodes
    from 2500 to 12000 K.  Returns (gencol dict, ecol, hcol): ecol / hcol mark the
    pairs whose electron / hydrogen rates the records supply."""
    rng = np.random.default_rng(seed + 5000)
    ion_lv = n - 1
    recs = [("CE", 0, 1), ("CE", 2, 5), ("CE", 3, 4), ("OHM", 4, 9), ("OHM", 8, 3), ("CH", 0, 1), ("CH", 5, 6),
            ("CI", 0, ion_lv), ("CI", 3, ion_lv), ("CHI", 1, ion_lv), ("CHI", 0, ion_lv), ("CH0", 2, ion_lv),
            ("UP", 2, 3), ("DN", 10 % nbound, 12 % nbound), ("NONE", 11 % nbound, 13 % nbound), ("CE", 0, 1)]
    recs = [r for r in recs if r[1] != r[2]]
    base = {"CE": -23.0, "OHM": -3.0, "CH": -31.0, "CI": -25.0, "CHI": -31.0, "CH0": -27.0, "UP": -29.0,
            "DN": -29.0, "NONE": -29.0}
    kinds = {"CE": 2, "OHM": 1, "CH": 3, "CHI": 4, "CI": 5, "CH0": 6, "UP": 7, "DN": 8, "NONE": 0}
    tgrid = np.geomspace(2500.0, 12000.0, ntemp)
    x = np.log(tgrid / 5000.0)
    lnc = np.zeros((len(recs), ntemp))
    for r, (key, _, _) in enumerate(recs):
        lnc[r] = base[key] + rng.uniform(0.2, 1.5) * x + 0.1 * np.sin(rng.uniform(1.0, 4.0) * x + rng.uniform(0, 6))
    lnc[1, 3:5] = lnc[1, 3]                # a flat stretch: zero slopes there
    lnc[2] = base["CE"] - 0.8 * x**2       # a turning point
    ecol = np.zeros((n, n), bool)
    hcol = np.zeros((n, n), bool)
    for key, l, u in recs:
        lo, hi = min(l, u), max(l, u)
        if key in ("CE", "CI", "OHM"):
            ecol[lo, hi] = True
        elif key in ("CH", "CHI", "CH0"):
            hcol[lo, hi] = True
    gc = {"tgrid": tgrid, "lnc": lnc, "ll": np.array([r[1] for r in recs], np.int32),
          "ul": np.array([r[2] for r in recs], np.int32), "kind": np.array([kinds[r[0]] for r in recs], np.int32),
          "collider": np.array([0 if r[0] == "UP" else 1 if r[0] == "DN" else -1 for r in recs], np.int32),
          "ch0_hmip": True}
    return gc, ecol, hcol


def _hydrogen_kinds(ion, col_i, col_j, col_fac, h_recipes):
    if not h_recipes:
        return None
    h_exc, h_ion, h_forb = h_recipes
    out = []
    for i, j, fac in zip(col_i, col_j, np.asarray(col_fac, np.float32)):
        cont = ion[j] > ion[i]
        if not cont and fac == 0 and h_forb == "takeda":
            out.append(2)
        elif (h_ion if cont else h_exc) == "drawin":
            out.append(1)
        else:
            out.append(0)
    return np.array(out, np.int32)


def hydrogen_ground(nH, ne):
    """A synthetic neutral hydrogen ground-level density: nH less the protons that
    charge neutrality with hydrogen as the only electron donor allows, at least 1%
    of nH."""
    nH = np.asarray(nH, np.float64)
    return nH * np.clip(1.0 - np.asarray(ne, np.float64) / nH, 0.01, 1.0)


def lte_populations(atom: dict, temp, ne, totn, dxi=None):
    """compute_lte_populations with the atom's own levels as partition function
    (level_partf, atom_mod.f90:1041-1140) and lte_pop (:1132-1150), in float64:
    returns nstar (nlevel, ncell) and totn = sum of nstar."""
    temp = np.asarray(temp, np.float64)
    ne = np.asarray(ne, np.float64)
    e_kT = (EE / BK) / temp
    lsaha = np.log(2.0 * (2.0 * PI * EM * BK * temp / HH**2) ** 1.5 / ne)
    dxi = np.zeros_like(temp) if dxi is None else np.asarray(dxi, np.float64)
    ion0 = atom["ion"][0]
    ns = np.empty((atom["nlevel"], temp.size))
    for i in range(atom["nlevel"]):
        j = atom["ion"][i]
        evi = atom["ev"][i] - dxi * 0.5 * (j - 1) * j
        tns = math.log(atom["g"][i]) - e_kT * evi + (j - ion0) * lsaha
        ns[i] = np.exp(tns)
    ns *= np.asarray(totn, np.float64) / ns.sum(axis=0)
    return ns, ns.sum(axis=0)


def se_inputs(atom: dict, temp, ne, nH, seed: int = 2, dilution=None, perturb: float = 0.3,
              abundance: float = 7.5) -> dict:
    """Per-cell inputs of one SE update (all (level or transition, cell), cell fastest):
    temp, ne, e_kT, nstar, totn, b (LTE times exp(N(0, perturb))), and the rates a
    diluted Planck field J = W B(T) gives: for a line th = g_j/g_i A_ji and
    dev = th n_ref (W - 1) (so R_ij = B_ij J, R_ji = A_ji + B_ji J in the
    (th, dev) form of line_rate_coefficients), for a continuum gamma_ij = W R0
    and gamma_ji = R0 n*_i/n*_j with R0 = 1e3/s.  W = 1 is LTE: detailed balance
    holds for every transition and b = 1 solves the rate equations."""
    rng = np.random.default_rng(seed + 3000)
    temp = np.ascontiguousarray(temp, np.float64).ravel()
    ne = np.ascontiguousarray(ne, np.float64).ravel()
    nH = np.ascontiguousarray(nH, np.float64).ravel()
    ncell = temp.size
    totn0 = 10.0 ** (abundance - 12.0) * nH
    nstar, totn = lte_populations(atom, temp, ne, totn0)
    e_kT = (EE / BK) / temp
    W = np.ones(ncell) if dilution is None else np.broadcast_to(np.asarray(dilution, np.float64), (ncell,))
    nrad, nline = len(atom["ti"]), atom["nline"]
    gij = np.zeros((nrad, ncell), np.float32)
    gji = np.zeros((nrad, ncell), np.float32)
    for kr in range(nrad):
        i, j = atom["ti"][kr], atom["tj"][kr]
        if kr < nline:
            hnu_kt = (atom["ev"][j] - atom["ev"][i]) * e_kT
            nref = 1.0 / np.expm1(hnu_kt)
            th = atom["g"][j] / atom["g"][i] * atom["Aji"][kr]
            gij[kr] = th
            gji[kr] = th * nref * (W - 1.0)
        else:
            gij[kr] = 1e3 * W
            gji[kr] = 1e3 * nstar[i] / nstar[j]
    b = np.exp(perturb * rng.standard_normal((atom["nlevel"], ncell))) if perturb > 0 else np.ones((atom["nlevel"], ncell))
    return {"temp": temp, "ne": ne, "e_kT": e_kT, "nstar": np.ascontiguousarray(nstar),
            "totn": np.ascontiguousarray(totn), "b": np.ascontiguousarray(b), "gamma_ij": gij, "gamma_ji": gji,
            "nh1": hydrogen_ground(nH, ne), "lsaha": lsaha(temp, ne),
            "colliders": np.ascontiguousarray(np.stack([0.1 * nH, 1e-3 * nH]))}


def lsaha(temp, ne):
    """comp%lsaha (composition_mod.f90:2423): ln(2 (2 pi m_e k / h^2)^(3/2) T^(3/2) / ne)."""
    temp = np.asarray(temp, np.float64)
    op_saha_const = (2 * math.pi * EM * BK / HH**2) ** 1.5
    return np.log(2 * op_saha_const * temp * np.sqrt(temp)) - np.log(np.asarray(ne, np.float64))


def se_config(kind: str = "small", seed: int | None = None, ncell: int | None = None, lte: bool = False,
              nbound: int = 20, nline: int = 60, h_recipes=None, gencol: bool = False) -> tuple:
    """(atom, inputs) of an SE case.  'c2': the 120^3 cube of seed 2 and the
    20-level atom with lines between levels at least 0.5 eV apart (a radiation
    field diluted upwards, W = exp(-3 z/nz));
    'small': ncell cells (default 2048) drawn from a 16^3 cube with W uniform
    in [0.05, 1]; lte: W = 1.  nbound/nline: the atom's bound levels and lines
    (60/180 for the larger atom of the batched configuration); h_recipes: the
    hydrogen collision recipes of model_atom; gencol: its tabulated records."""
    if kind == "c2":
        seed = 2 if seed is None else seed
        cube = cube_atmosphere(seed, 120, 120, 120)
        nz = 120
        W = np.exp(-3.0 * (np.arange(nz) + 0.5) / nz)[:, None, None] * np.ones((1, 120, 120))
    elif kind == "small":
        seed = 5 if seed is None else seed
        cube = cube_atmosphere(seed, 16, 16, 16)
        W = np.random.default_rng(seed + 4000).uniform(0.05, 1.0, 16**3)
    else:
        raise ValueError(kind)
    atom = model_atom(seed, nbound=nbound, nline=nline, h_recipes=h_recipes, gencol=gencol,
                      min_line_ev=0.5 if kind == "c2" else 0.0)
    temp, ne, nH = cube["temp"].ravel(), cube["ne"].ravel(), cube["nH"].ravel()
    W = np.asarray(W).ravel()
    if ncell is not None:
        idx = np.arange(ncell) % temp.size
        temp, ne, nH, W = temp[idx], ne[idx], nH[idx], W[idx]
    return atom, se_inputs(atom, temp, ne, nH, seed=seed, dilution=None if lte else W)


def _set_weights(x):
    """set_weights (HOP/spectrum_mod.f90:491-513): trapezoid weights, positive."""
    x = np.asarray(x, np.float64)
    w = np.empty_like(x)
    if x.size == 1:
        return np.ones(1)
    w[0] = 0.5 * (x[1] - x[0])
    w[1:-1] = 0.5 * (x[2:] - x[:-2])
    w[-1] = 0.5 * (x[-1] - x[-2])
    return np.abs(w)


def atom_window(atom: dict, nper: int = 25, seed: int = 2, qmax_doppler: float = 5.0, idf_ref: float = 1.8e5,
                adamp=(1e-3, 1e-1), sums=None, transitions=None, lam_range=None) -> dict:
    """The atom's transitions on one frequency window holding every transition:
    nper points per line on q = 1 - lam/lam0 in +-qmax_doppler/idf_ref, nper
    points per continuum from 0.3 of its edge wavelength to the edge, merged
    into one grid ascending in wavelength.  A transition's window is every grid
    point inside its own range (the reference's get_interval), with q, the rate
    weights wnu (set_weights in nu, / nu for a line, / (h/4pi nu) for a
    continuum) and the profile weights wq over all of them.  Lines: Einstein
    coefficients of init_einstein_coefficients (bbtrans_mod.f90:55-67) from the
    atom's f values, damping a log-uniform in adamp (grad = a/idf_ref), no van der
    Waals or Stark terms; continua: Kramers-shaped alpha0 (lam/lam_edge)^3.
    sums: per line sums_over_windows (default none).  transitions: the atom's
    transition indices the window holds (default all), the reference's split of
    the spectrum into frequency windows; a transition keeps its damping in every
    window.  lam_range: (lo, hi) [AA], a window by wavelength instead -- the grid's
    points in [lo, hi), every transition with points there, a transition that
    straddles the bounds keeping only its part (the reference's contiguous
    n_windows chunks, where a continuum can span several windows)."""
    rng = np.random.default_rng(seed + 5000)
    nline = atom["nline"]
    ti, tj, ev, g = atom["ti"], atom["tj"], atom["ev"], atom["g"]
    nrad = len(ti)
    lam_pts = []
    q0 = np.linspace(-qmax_doppler / idf_ref, qmax_doppler / idf_ref, nper)
    lam0 = np.array([HH * CC / ((ev[tj[k]] - ev[ti[k]]) * EE) * 1e8 for k in range(nrad)])
    ks = list(range(nrad)) if transitions is None else sorted(int(k) for k in transitions)
    for k in range(nrad):
        if k < nline:
            lam_pts.append(lam0[k] * (1.0 - q0))
        else:
            lam_pts.append(np.geomspace(0.3 * lam0[k], lam0[k] * (1.0 - 1e-7), nper))
    grid = np.unique(np.concatenate([lam_pts[k] for k in ks]))
    if lam_range is not None:
        grid = grid[(grid >= lam_range[0]) & (grid < lam_range[1])]
        ks = [k for k in ks if np.any((lam_pts[k] >= lam_range[0]) & (lam_pts[k] < lam_range[1]))]
        lam_pts = [p[(p >= lam_range[0]) & (p < lam_range[1])] for p in lam_pts]
    nu = HZ_TO_AA / grid
    nf = grid.size
    li, lj, lb, lr, lo, q, wnu, wq = [], [], [], [], [], [], [], []
    ci, cj, cb, cr, co, alpha, cwnu = [], [], [], [], [], [], []
    off_l = off_c = 0
    f_osc = atom.get("line_f", np.full(nline, 0.1))
    Aij, Bij, lk = [], [], []
    for k in ks:
        lo_lam, hi_lam = lam_pts[k].min(), lam_pts[k].max()
        blue = int(np.searchsorted(grid, lo_lam, "left"))
        red = int(np.searchsorted(grid, hi_lam, "right")) - 1
        sl = slice(blue, red + 1)
        if k < nline:
            nu0 = CC / (lam0[k] * 1e-8)
            Aij.append(F_CONV * f_osc[k] * nu0**2)
            Bij.append(C2_2H / nu0**3 * (Aij[-1] * H_4PI))
            lk.append(k)
            qq = (1.0 - grid[sl] / lam0[k]).astype(np.float32)
            li.append(ti[k]); lj.append(tj[k]); lb.append(blue); lr.append(red); lo.append(off_l)
            q.append(qq)
            wnu.append(_set_weights(nu[sl]) / nu[sl])
            wq.append(_set_weights(qq.astype(np.float64)))
            off_l += red - blue + 1
        else:
            a0 = 7.91e-18 * math.sqrt(RYDV / (ev[tj[k]] - ev[ti[k]]))
            ci.append(ti[k]); cj.append(tj[k]); cb.append(blue); cr.append(red); co.append(off_c)
            alpha.append((a0 * (grid[sl] / lam0[k]) ** 3).astype(np.float32))
            cwnu.append(_set_weights(nu[sl]) / (H_4PI * nu[sl]))
            off_c += red - blue + 1
    a = 10.0 ** rng.uniform(math.log10(adamp[0]), math.log10(adamp[1]), nline)
    sums = np.zeros(nline, np.uint8) if sums is None else np.asarray(sums, np.uint8)
    lk = np.asarray(lk, np.int64)
    nl = lk.size
    ck = [k for k in ks if k >= nline]
    i32 = lambda v: np.asarray(v, np.int32)
    cat = lambda v, dt: np.concatenate(v).astype(dt) if v else np.zeros(0, dt)
    return {"nf": nf, "lam": grid, "nu": nu, "nline": nl, "ncont": len(ck), "nlevel": atom["nlevel"],
            "line_i": i32(li), "line_j": i32(lj), "line_ntrans": i32(lk),
            "line_index": i32(lk + 1), "line_blue": i32(lb), "line_red": i32(lr), "line_off": i32(lo),
            "q": cat(q, np.float32), "wnu": cat(wnu, np.float64), "wq": cat(wq, np.float64),
            "Bij": np.asarray(Bij, np.float64), "Aij": np.asarray(Aij, np.float64),
            "lower_ev": np.asarray(ev[ti[lk]], np.float64),
            "line_active": None, "sums_over_windows": sums[lk],
            "grad": a[lk] / idf_ref, "gw1": np.zeros(nl), "gw2": np.zeros(nl), "gstk": np.zeros(nl),
            "unsold": np.zeros(nl, np.uint8),
            "cont_i": i32(ci), "cont_j": i32(cj), "cont_ntrans": i32(ck),
            "cont_blue": i32(cb), "cont_red": i32(cr), "cont_off": i32(co),
            "alpha": np.concatenate(alpha).astype(np.float32) if alpha else np.zeros(0, np.float32),
            "cwnu": np.concatenate(cwnu) if cwnu else np.zeros(0),
            "cont_active": None, "g": np.asarray(g, np.float64), "ev": np.asarray(ev, np.float64), "cut_x": 70.0,
            "twohnu3_c2": (2.0 * HH * nu**3 / CC**2).astype(np.float32)}


def pca_grid(temp, ne, ldtemp=0.05, ldne=0.25, npad=2):
    """An orthogonal PC basis of (ln T, ln ne) over the given cells and a regular
    node grid along its axes (the pca_transform_type of optab_mod.f90:26-31):
    mu the mean, rot the unit eigenvectors as columns (largest variance first,
    first component of each made positive), c0 the first node and dc the spacing
    (the requested ln T / ln ne steps projected onto each axis), npad nodes past
    the data at either end.  Returns (pca dict, n1, n2)."""
    x = np.stack([np.log(np.asarray(temp, np.float64).ravel()), np.log(np.asarray(ne, np.float64).ravel())])
    mu = x.mean(axis=1)
    w, v = np.linalg.eigh(np.cov(x))
    rot = v[:, ::-1].copy()
    rot *= np.sign(rot[0])[None, :]
    p = rot.T @ (x - mu[:, None])
    step = np.array([ldtemp, ldne])
    dc = np.array([1.0 / np.sqrt(np.sum((rot[:, k] / step) ** 2)) for k in range(2)])
    c0 = p.min(axis=1) - npad * dc
    n = np.floor((p.max(axis=1) - c0) / dc).astype(int) + 1 + npad
    return {"mu": mu, "rot": rot, "c0": c0, "dc": dc}, int(n[0]), int(n[1])


def table_nodes(pca, n1, n2):
    """(T, ne) at the PC grid nodes, (n2, n1) each (pca_opac_grid, optab_mod.f90:515-523)."""
    i = np.arange(n1)[None, :]
    j = np.arange(n2)[:, None]
    p1 = pca["c0"][0] + i * pca["dc"][0]
    p2 = pca["c0"][1] + j * pca["dc"][1]
    r = np.asarray(pca["rot"])
    lnT = pca["mu"][0] + r[0, 0] * p1 + r[0, 1] * p2
    lnN = pca["mu"][1] + r[1, 0] * p1 + r[1, 1] * p2
    return np.exp(lnT), np.exp(lnN)


def sample_table(seed, temp, ne, nnu=800, lam=(4000.0, 9000.0), kind="background", scat=True, ldtemp=0.05,
                 ldne=0.25, npad=2, nline=40, lam_nodes=None):
    """A synthetic sampled opacity table over the (T, ne) of the given cells: an
    irregular ascending wavelength grid, the PC node grid of pca_grid, and a
    positive opacity per unit chi500 on it.  kind "background": a smooth H- like
    continuum with edges plus, as the scattering component, a Rayleigh-like
    lambda^-4 term; kind "linelist": nline Lorentzian lines whose strengths follow
    Boltzmann factors of the node temperatures, with (1-eps) = 0.3 of each as the
    scattering component.  lam_nodes, when given, are the wavelength nodes (the
    reference tabulates on the window's own frequencies, rt_patch_mod.f90:2359,
    padded for Doppler shifts on the line-list path, :2440-2466).  Returns a
    dict: lam (nnu,), val and scat (nne, ntemp, nnu) or scat None, pca."""
    rng = np.random.default_rng(seed)
    pca, n1, n2 = pca_grid(temp, ne, ldtemp, ldne, npad)
    if lam_nodes is not None:
        lam_n = np.asarray(lam_nodes, np.float64)
        lam = (float(lam_n[0]), float(lam_n[-1]))
    else:
        u = np.sort(rng.random(nnu - 2))
        lam_n = np.concatenate([[lam[0]], lam[0] * (lam[1] / lam[0]) ** u, [lam[1]]])
        lam_n = np.unique(lam_n)
        while lam_n.size < nnu:
            lam_n = np.unique(np.concatenate([lam_n, [lam_n[0] + (lam_n[1] - lam_n[0]) * 0.5]]))
    Tn, Nn = table_nodes(pca, n1, n2)
    th = 5040.0 / Tn[:, :, None]
    L = lam_n[None, None, :] / 5000.0
    if kind == "background":
        cont = (Nn[:, :, None] / 1e14) ** 0.8 * np.exp(-0.75 * th) * L ** 1.5
        edges = sum(a * (L > e) * L ** 3 for a, e in ((0.6, 0.82), (0.3, 1.3), (0.2, 1.65)))
        val = cont * (1.0 + edges) * (1.0 + 0.05 * np.sin(7.0 * L))
        sc = 0.02 * L ** -4 * (1.0 + 0.5 * th) * np.ones_like(val)
    else:
        val = np.zeros((n2, n1, lam_n.size))
        l0 = rng.uniform(lam[0], lam[1], nline)
        w = rng.uniform(0.05, 0.3, nline)
        chi_ex = rng.uniform(0.0, 4.0, nline)
        s0 = 10.0 ** rng.uniform(-1.0, 2.0, nline)
        for k in range(nline):
            prof = w[k] ** 2 / ((lam_n - l0[k]) ** 2 + w[k] ** 2)
            val += s0[k] * 10.0 ** (-chi_ex[k] * th) * prof[None, None, :]
        sc = 0.3 * val
    out = {"lam": lam_n, "val": val.astype(np.float32), "pca": pca}
    out["scat"] = sc.astype(np.float32) if scat else None
    return out


def optab_cells(seed, nx, ny, nz):
    """Cell temperatures, electron densities, chi500 and projected velocities
    (v/c) of a seeded cube, flat (nz*ny*nx,), with ne tied to T as well as to the
    density so that (ln T, ln ne) spread about their principal axis."""
    atm = cube_atmosphere(seed, nx, ny, nz)
    T = atm["temp"].astype(np.float64)
    ne = atm["ne"] * np.exp((T - 6000.0) / 1500.0)
    return {"temp": T.ravel(), "ne": ne.ravel(), "chi500": atm["chi_c"].ravel().astype(np.float32),
            "vproj": atm["vz"].ravel().astype(np.float32)}


def window_tables(seed, temp, ne, vproj, nf=256, lam0=5040.0, R=1e5, pad_guard=2, nline=30):
    """The two tables of one frequency window as the reference builds them: the
    window's nf wavelengths uniform in ln lambda at resolution R (lam_q); the
    background table on exactly those nodes (rt_patch_mod.f90:2359); the line-list
    table on them extended by ceil(vmax / dlnlam) + pad_guard nodes at either end
    (:2440-2466), vmax the largest |vproj|.  Returns (lam_q, background, linelist)."""
    dl = 1.0 / R
    lam_q = lam0 * np.exp(dl * np.arange(nf))
    vmax = float(np.max(np.abs(vproj))) if np.size(vproj) else 0.0
    npad = int(np.ceil(vmax / dl)) + pad_guard
    plam = lam0 * np.exp(dl * np.arange(-npad, nf + npad))
    plam[npad:npad + nf] = lam_q
    bg = sample_table(seed, temp, ne, kind="background", lam_nodes=lam_q)
    ll = sample_table(seed + 1, temp, ne, kind="linelist", lam_nodes=plam, nline=nline)
    return lam_q, bg, ll


def continuum_case(seed: int = 5, ncell: int = 2000, nlam: int = 256, lam_range=(3500.0, 12000.0)) -> tuple:
    """(comps, lam, nu, cells) of a seeded continuum-opacity case: fourteen absdat-like
    components, one or more of every absorption-factor kind (two 'H BF' levels under
    occupation probabilities among them), their tables in the
    stored form of set_table (dispatch_b200.continuum.set_table) with every
    interpolation choice -- linear or quadratic in temperature (T or 5040/T nodes),
    logarithmic tables, linear, quadratic or logarithmic in wavelength, nodes flagged
    as discontinuities, extrapolation allowed or not at each end, lam^3 scaling, no
    temperature dependence -- two tabulated with stimulated emission; tables that
    cover the window only in part; cells below, inside and above the temperature
    nodes; the EOS state drawn from a grey-atmosphere-like range (T 3500-12000 K,
    ne 1e10-1e15 cm^-3).  The tables are synthetic (smooth positive cross sections
    of realistic size), not HOP's absdat data."""
    from .continuum import (H, H2PLUS, H_FF, HMINUS, MOLECULAR, NPE, PAIR, PEACH, PEDEP, REGULAR, set_table)
    rng = np.random.default_rng(seed + 7000)
    lam = np.geomspace(lam_range[0], lam_range[1], nlam)
    nu = HZ_TO_AA / lam
    temp = rng.uniform(3500.0, 12000.0, ncell)
    e_kT = EE / (BK * temp)
    ne = 10.0 ** rng.uniform(10.0, 15.0, ncell)
    cells = {"temp": temp, "teta": 5040.0 / temp, "e_kT": e_kT, "pe": ne * BK * temp,
             "dxi": rng.uniform(0.0, 0.06, ncell), "ne": ne, "nHI": 10.0 ** rng.uniform(14.0, 17.0, ncell),
             "partHI": np.log(2.0) + rng.uniform(0.0, 1e-3, ncell), "nHeI": 10.0 ** rng.uniform(13.0, 16.0, ncell),
             "nH2": 10.0 ** rng.uniform(6.0, 12.0, ncell), "HI_xion": 13.598434, "helium_scattering": True}
    dens = lambda lo, hi: 10.0 ** rng.uniform(lo, hi, ncell)

    def table(kind, nnu, lrange, tnodes, shape, ilogt=False, ilogl=False, **kw):
        tl = np.geomspace(lrange[0], lrange[1], nnu)
        tt = np.asarray(tnodes, np.float64)
        raw = np.array([[shape(l, t) for l in tl] for t in tt]) if tt.size > 1 else np.array([[shape(l, 6000.0)
                                                                                               for l in tl]])
        xk, scale, logt = set_table(raw, ilogt, ilogl)
        ld = np.zeros(nnu, bool)
        ld[rng.choice(nnu - 2, size=max(1, nnu // 12), replace=False) + 1] = True
        c = {"kind": kind, "lam": tl, "tt": tt, "xkap": xk, "xkap_scale": scale, "log_table": logt, "ldisk": ld,
             "ilogl": ilogl, "minl": tl[0], "maxl": tl[-1], "mint": 0.0, "maxt": 1e9}
        c.update(kw)
        return c

    tnod = np.linspace(4000.0, 10000.0, 7)
    teta_nod = np.sort(5040.0 / np.linspace(4500.0, 11000.0, 8))
    sig = lambda a, p: (lambda l, t: a * (l / 5000.0) ** p * (1.0 + 0.3 * np.sin(l / 700.0)) * (t / 6000.0) ** 0.5)
    comps = [
        table(HMINUS, 40, (2500.0, 16000.0), teta_nod, sig(4e-17, 0.8), ilogt=True, iteta=True, kvadl=True,
              n=dens(8.0, 10.5)),
        table(NPE, 30, (3000.0, 20000.0), tnod, sig(2e-26, 2.0), ilogt=True, kvadt=True, maxex=True,
              n=dens(14.0, 17.0)),
        table(H, 50, (3000.0, 8205.0), [6000.0], lambda l, t: 1e-17 * (l / 8205.0) ** 3, ilogl=True, lam3=True,
              kvadl=True, k=3, level_n=dens(2.0, 7.0)),
        table(H_FF, 20, (2000.0, 25000.0), tnod[:5], sig(1e-12, 1.0), lam3=True, ion_xion=13.598434,
              n=dens(9.0, 13.0), part=np.log(rng.uniform(1.0, 1.5, ncell))),
        table(PAIR, 25, (4000.0, 30000.0), [3000.0, 5000.0, 7000.0, 9000.0], sig(1e-45, 1.5), ilogt=True,
              ilogl=True, loglam=True, n=dens(14.0, 17.0), n2=dens(13.0, 16.0)),
        table(H2PLUS, 18, (3800.0, 9000.0), [4500.0, 6000.0, 7500.0], sig(1e-5, 0.5), kvadt=True,
              mint=4600.0, maxt=9000.0, n=dens(10.0, 14.0), n2=dens(8.0, 12.0)),
        table(PEDEP, 45, (3500.0, 11000.0), [5000.0], sig(3e-27, 1.2), kvadl=True, minex=True, maxex=True,
              n=dens(8.0, 12.0)),
        table(PEACH, 35, (3200.0, 13000.0), teta_nod[:7], sig(5e-3, 0.7), ilogt=True, iteta=True, kvadt=True,
              kvadl=True, n=dens(6.0, 11.0)),
        table(MOLECULAR, 22, (5000.0, 15000.0), tnod[1:], sig(2e-3, 1.0), ilogl=True, kvadt=True, minex=True,
              awgt=28.0, n=dens(6.0, 10.0)),
        table(REGULAR, 28, (3500.0, 7000.0), [6000.0], sig(2e-18, 3.0), lam3=True, level_g=9.0, level_xion=3.2,
              n=dens(10.0, 13.0), part=np.log(rng.uniform(5.0, 30.0, ncell))),
        table(HMINUS, 32, (4000.0, 14000.0), tnod, sig(3e-17, 0.6), istim=True, kvadt=True, kvadl=True,
              loglam=True, n=dens(8.0, 10.5)),
        table(REGULAR, 26, (3000.0, 9000.0), tnod[::2], sig(1e-18, 2.0), istim=True, ilogt=True, lam3=True,
              level_g=2.0, level_xion=1.1, minex=True, n=dens(10.0, 13.0), part=np.log(rng.uniform(2.0, 9.0, ncell))),
    ]
    # two 'H BF' levels under occupation probabilities (the reference's default),
    # n = 2 and 3: Gaunt-factor-like tables (2.0898e-26/(2 n^5) lam^3 is Kramers'
    # cross section) up to the series limit, extrapolated beyond it (maxex, as
    # the reference sets for these levels); the window then holds wavelengths beyond
    # each limit, dissolved upper states below it (both perturber branches of wcalc2,
    # w near 1), and the cut past the alpha line
    cells["shield"] = h_shield(temp, ne)
    for i, dissolved in ((2, False), (3, True)):
        edge = 911.267 * i * i
        xion = 13.598434 * float(np.float32(1.0) - np.float32(1.0) / np.float32(i * i))
        g = 2.0 * i * i
        lvl_n = g * np.exp(-e_kT * xion) * cells["nHI"] / 2.0
        w = h_occupation(cells["nHI"], cells["nHeI"], ne, cells["shield"], float(i))
        c = table(H, 16 + 2 * i, (600.0, edge), [6000.0], lambda l, t: 0.95 * (l / edge) ** 0.1, lam3=True,
                  kvadl=True, maxex=True, occupation=True, level_i=i, level_xion=xion, k=i, n=cells["nHI"],
                  level_n=lvl_n, level_w=w, dissolved_only=dissolved)
        comps.append(c)
    return comps, lam, nu, cells


def h_shield(temp, ne):
    """composition_type%compute_shield (HOP/composition_mod.f90:2604-2613): the
    charged-perturber shielding (1 + a)^3.15 / ne, a = 0.08989 ne^(1/6) / sqrt(T)."""
    a = 0.08989 * np.asarray(ne) ** 0.16667 / np.sqrt(np.asarray(temp))
    return (1.0 + a) ** 3.15 / np.asarray(ne)


def h_occupation(nh, nhe, ne, shield, ns):
    """wcalc (HOP/level_mod.f90:108-142): the occupation probability of an H I state
    of effective quantum number ns -- hard-sphere neutral H and He perturbers
    (Hummer & Mihalas 1988) times the charged-perturber fit of Hubeny, Hummer & Lanz
    (1994) where k x < 1e4.  A numpy stand-in for the EOS's level set-up."""
    ns2 = ns * ns
    rih = ns * np.sqrt(2.5 * ns2 + 0.5)
    x1 = (5.29177349e-9 * (rih + 1.73)) ** 3
    x2 = (5.29177349e-9 * (rih + 1.02)) ** 3
    k = 8.3e14 / (ns2 * ns2)
    if ns > 3.0:
        k = k * 5.33333333 * ns / (ns + 1.0) ** 2
    k = k * np.sqrt(k)
    res = np.exp(-4.18879 * (np.asarray(nh) * x1 + np.asarray(nhe) * x2))
    x = np.asarray(shield)
    charged = k * x < 1e4
    frac = 0.1402 * x * k * k / (np.asarray(ne) * (1.0 + 0.1285 * x * k))
    return np.where(charged, res * frac / (1.0 + frac), res)

"""The hydrogen line-profile oracle (oracle/or_hprof.c) and the library's host-side
hydrogen_line.  The reference has no golden vectors for these profiles; its own
statements are the pins: unit area in a Doppler-dominated cell (hvoigt's
components are unit-area Voigt profiles with weights summing to one,
hprofl_mod.f90:460-499), and a Lyman line redward of 1400 A adding only roundoff
in a cool thin cell (HOP/tests/test_hop.py, test_lyman_wing_gives_way_to_rayleigh_
scattering).  The walk of add_h_opacities is checked point by point against the
profile."""
import numpy as np
import pytest

import hprof_cases as hc


def test_library_hydrogen_line_equals_oracle(m3d_lib, oracle):
    from dispatch_b200 import hprof as dh
    from oracle import hprof as oh
    for n, m, lam in hc.LINES + [(2, 30, 3663.4), (6, 7, 123720.0), (1, 11, 918.1)]:
        for opts in (0, 1, 2, 4, 8, 15):
            a = dh.hydrogen_line(n, m, hc.nu0(lam), opts)
            b = oh.hydrogen_line(n, m, hc.nu0(lam), opts)
            assert bytes(a) == bytes(b), (n, m, opts)
    h = dh.hydrogen_line(2, 3, hc.nu0(6564.61))
    assert h.bpo == 1 and h.io == 7 and abs(sum(h.wt[:7]) - 1.0) < 1e-6
    with pytest.raises(m3d_lib.M3DError, match="n < m"):
        dh.hydrogen_line(3, 3, 1e15)


@pytest.mark.parametrize("n,m,lam", [(1, 2, 1215.668), (2, 3, 6564.61), (3, 4, 18756.1), (2, 12, 3751.2)])
def test_unit_area_when_doppler_dominated(oracle, n, m, lam):
    from oracle import hprof as oh
    h = oh.hydrogen_line(n, m, hc.nu0(lam))
    cell = {"temp": 6000.0, "ne": 1e9, "tothi": 1e12, "fo": 1.25e-9 * 1e6, "vbar2h": 1e11, "t3nhe": 1e10,
            "inv_df": 2.99792458e10 / 1.1e6}
    q = np.concatenate([-np.logspace(-0.5, -10, 12000), [0.0], np.logspace(-10, -0.5, 12000)])
    phi = oh.hprofile(h, cell, q).astype(np.float64)
    assert np.trapezoid(phi, q) == pytest.approx(1.0, abs=5e-3)      # far wings past |q| = 0.32 left out


def test_lyman_beta_red_of_1400_is_roundoff(oracle):
    from oracle import hprof as oh
    h = oh.hydrogen_line(1, 3, hc.nu0(1025.722))
    cell = {"temp": 3800.0, "ne": 1e8, "tothi": 1e13, "fo": 1.25e-9 * 1e8 ** (2 / 3), "vbar2h": 1e11,
            "t3nhe": 1e12, "inv_df": 2.99792458e10 / 8e5}
    lam = np.array([1030.0, 1100.0, 1399.0, 1401.0, 2000.0, 10000.0])
    q = hc.nu0(lam) / hc.nu0(1025.722) - 1.0
    phi = oh.hprofile(h, cell, q)
    peak = oh.hprofile(h, cell, np.array([0.0]))[0]
    assert (phi[lam > 1400] / peak < 1e-12).all()
    assert phi[0] / peak > 1e-9                      # blueward the natural wing is kept


def test_walk_adds_the_profile_until_below_tolerance(oracle):
    from oracle import hprof as oh
    c = hc.cells(seed=4, n=9)
    for n, m, lam in [(2, 3, 6564.61), (1, 2, 1215.668)]:
        nu = hc.grid(lam, 40.0 if n == 2 else 8.0, 801)
        f0 = int(np.argmin(np.abs(nu - hc.nu0(lam))))
        h = oh.hydrogen_line(n, m, hc.nu0(lam))
        cont = np.full((9, 801), 1e-9, np.float32)
        chi = np.zeros((9, 801), np.float32)
        eta = np.zeros((9, 801), np.float32)
        used, strength = oh.add_h_opacities(h, 1e-8, f0, nu, c, chi, eta, cont)
        assert used and strength > 0
        np.testing.assert_array_equal(chi, eta)                 # LTE: no departure coefficients
        for i in range(9):
            cell = {k: float(c[k][i]) for k in c}
            v = np.float32((np.float64(np.float32(c["vproj"][i] + np.float32(1.0))) * h.nu0))
            q = (nu - np.float64(v)) * np.float64(np.float32(1.0 / h.nu0))
            cchi = np.float32(np.float64(c["ni"][i]) * 1e-8)
            want = oh.hprofile(h, cell, q) * cchi
            got = chi[i]
            nz = np.nonzero(got)[0]
            assert nz[0] <= f0 <= nz[-1] and np.all(np.diff(nz) == 1)
            np.testing.assert_array_equal(got[nz], want[nz])
            ref = np.float32(1e-7) * cont[i, f0]
            assert want[nz[-1]] < ref or nz[-1] == 800
            assert want[nz[0]] < ref or nz[0] == 0
            assert (want[nz[0] + 1:f0] >= ref).all() and (want[f0:nz[-1]] >= ref).all()


def _load_synthetic(tmp_path, oh):
    import vcs_cases
    paths = vcs_cases.write_all(str(tmp_path))
    for s, p in paths.items():
        oh.vcs_load(s, p, s == 3)
    return paths


def test_vcs_profile_is_normalised_and_continues_into_its_tail(oracle, tmp_path):
    """The prepared table profile has unit area under the trapezium rule
    vcs_cell_profile normalises with, and the power-law tail meets vcs_eval at the
    table's outer edge (tail_coef extrapolates qpol's log-log line there)."""
    from oracle import hprof as oh
    _load_synthetic(tmp_path, oh)
    try:
        for n, m, lam in [(2, 3, 6564.61), (2, 12, 3751.2), (3, 4, 18756.1), (4, 7, 21661.2)]:
            h = oh.hydrogen_line(n, m, hc.nu0(lam))
            for T, ne, nH in [(4500.0, 3e11, 1e15), (9000.0, 5e14, 1e13), (20000.0, 1e17, 1e17)]:
                cell = {"temp": T, "ne": ne, "tothi": nH, "fo": 1.25e-9 * ne ** (2 / 3), "vbar2h": 1e11,
                        "t3nhe": 1e10, "inv_df": 2.99792458e10 / 1.1e6}
                lam0 = lam
                q_edge = 10 ** (-2.0 + 4.3) / lam0
                q = np.array([q_edge * (1 - 1e-7), q_edge * (1 + 1e-7), -q_edge * (1 - 1e-7)])
                # the tail's own branch starts past q_edge + dqmax; close to it both sides agree
                phi = oh.hprofile(h, cell, q)
                assert phi[0] == pytest.approx(phi[1], rel=2e-3)
                # unit area in q over the table (trapezium over a fine grid, both wings)
                qq = np.concatenate([-np.logspace(np.log10(q_edge), -9, 6000), np.logspace(-9, np.log10(q_edge), 6000)])
                area = np.trapezoid(oh.hprofile(h, cell, qq).astype(np.float64), qq)
                assert 0.9 < area < 1.05
    finally:
        oh.vcs_clear()


def test_vcs_reads_the_reference_tables_when_present(oracle):
    """With the reference's own table files at hand (not on every machine), every
    series loads and every tabulated Balmer line gives a finite, positive profile."""
    import os
    from oracle import hprof as oh
    ref = os.environ.get("M3D_REFERENCE_ROOT", "")   # the reference's experiments/OpenMULTI3D tree
    d = os.path.join(ref, "HOP", "hopacity", "data", "vcs")
    if not ref or not os.path.isdir(d):
        pytest.skip("the reference's VCS tables are not present")
    try:
        oh.vcs_load(1, os.path.join(d, "stehle_balmer.txt"), False)
        oh.vcs_load(2, os.path.join(d, "stehle_paschen.txt"), False)
        oh.vcs_load(3, os.path.join(d, "vcs_bracket.txt"), True)
        q = np.linspace(-1e-3, 1e-3, 101)
        for m in range(3, 12):
            h = oh.hydrogen_line(2, m, 2.99792458e18 / (911.5 / (0.25 - 1.0 / m ** 2) / 4))
            phi = oh.hprofile(h, {"temp": 6000.0, "ne": 1e14, "tothi": 1e16, "fo": 1.25e-9 * 1e14 ** (2 / 3),
                                  "vbar2h": 1e11, "t3nhe": 1e14, "inv_df": 2.99792458e10 / 1.1e6}, q)
            assert np.isfinite(phi).all() and phi.min() > 0
    finally:
        oh.vcs_clear()

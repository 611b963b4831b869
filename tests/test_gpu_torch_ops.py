"""torch.ops.m3d against the ctypes front end: the same C ABI behind both, so every
operator's results equal the front end's bit for bit, on torch's current stream."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops(m3d):
    from dispatch_b200 import torch_ops
    return torch_ops.load()


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _datm(atm):
    d = {k: (_dev(v) if isinstance(v, np.ndarray) and k != "slab_nz" else v) for k, v in atm.items()}
    d["species"] = [{k: _dev(v) for k, v in sp.items()} for sp in atm["species"]]
    return d


def test_lte_ops_match_front_end(m3d, ops):
    import torch
    from dispatch_b200 import synth, torch_ops
    atm, nu, llam, vec, wmu = synth.lte_config("mini", nf=32, window=5)
    ie, flux, itop = m3d.lte_synthesis(atm, nu, llam, vec, wmu, return_itop=True)
    datm = _datm(atm)
    tie, tflux, titop = torch_ops.lte_synthesis(datm, _dev(nu), _dev(llam), vec, wmu, return_itop=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(tie.cpu().numpy(), ie)
    np.testing.assert_array_equal(tflux.cpu().numpy(), flux)
    np.testing.assert_array_equal(titop.cpu().numpy(), itop)
    for fp64 in (False, True):
        chi, S = m3d.lte_transfer_units(atm, nu, llam, vec[4], fp64=fp64)
        tchi, tS = torch_ops.lte_transfer_units(datm, _dev(nu), _dev(llam), vec[4], fp64=fp64)
        np.testing.assert_array_equal(tchi.cpu().numpy(), chi)
        np.testing.assert_array_equal(tS.cpu().numpy(), S)
    rng = np.random.default_rng(3)
    g_flux = rng.uniform(0.5, 1.5, nu.size).astype(np.float32)
    g = m3d.lte_synthesis_adjoint(atm, nu, llam, vec, wmu, g_flux)
    tg = torch_ops.lte_synthesis_adjoint(datm, _dev(nu), _dev(llam), vec, wmu, _dev(g_flux))
    for k in g:
        np.testing.assert_allclose(tg[k].cpu().numpy().reshape(g[k].shape), g[k], rtol=1e-5,
                                   atol=1e-6 * np.abs(g[k]).max())   # atomic sums: order may differ


def test_solver_ops_match_front_end(m3d, ops, oracle):
    import torch
    from test_gpu_parity import _slab_case
    nf, nx, ny, nz = 8, 12, 10, 6
    vec = np.array([0.31, -0.22, 0.0])
    vec[2] = math.sqrt(1 - (vec[:2] ** 2).sum())
    ds = [1.2e7, 1.0e7, 0.8e7]
    work, c5, c5u, g5, er, em = _slab_case(17, nf, nx, ny, nz, np.float32, vec)
    for solver in ("QUADRATIC", "SHORT_LINEAR"):
        w = work.copy()
        psi = np.zeros((nz, ny, nx, nf), np.float32)
        slab = m3d.make_slab(nf, nx, ny, nz, 1, ds, vec, get_psi=True)
        rot = ((0.12, 0.1, 0.08), 1.7, (0.25, -0.5)) if solver == "QUADRATIC" else None
        m3d.formal_solve(getattr(m3d, solver), slab, w, psi=psi, rotate=rot)
        tw, tpsi = _dev(work), _dev(np.zeros((nz, ny, nx, nf), np.float32))
        ops.formal_solve(getattr(m3d, solver), tw, tpsi, None, None, None, None, None, None, None,
                         [nf, nx, ny, nz], 1, ds, [float(v) for v in vec], True, False, 2.0, 1e30,
                         None if rot is None else list(rot[0]) + [rot[1]] + list(rot[2]))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(tw.cpu().numpy(), w)
        np.testing.assert_array_equal(tpsi.cpu().numpy(), psi)
    # rotate_array, integrate_intensity, the QLG-bot profile
    w = work.copy()
    m3d.rotate_array(m3d.make_slab(nf, nx, ny, nz, 1, [1.0] * 3, vec), w, (0.12, 0.1, 0.08), 2.3, (0.0, 0.5))
    tw = _dev(work)
    ops.rotate_array(tw, [nf, nx, ny, nz], [float(v) for v in vec], [0.12, 0.1, 0.08], 2.3, [0.0, 0.5])
    np.testing.assert_array_equal(tw.cpu().numpy(), w)
    rng = np.random.default_rng(5)
    inu, psi = rng.uniform(0, 2, 500).astype(np.float32), rng.uniform(0, 1, 500).astype(np.float32)
    J, P = rng.uniform(0, 1, 500).astype(np.float32), rng.uniform(0, 1, 500).astype(np.float32)
    tJ, tP = _dev(J), _dev(P)
    m3d.integrate_intensity(0.0833, inu, psi, J, P)
    ops.integrate_intensity(0.0833, _dev(inu), _dev(psi), tJ, tP)
    np.testing.assert_array_equal(tJ.cpu().numpy(), J)
    np.testing.assert_array_equal(tP.cpu().numpy(), P)
    a = rng.uniform(1e-3, 0.1, 300).astype(np.float32)
    q = rng.uniform(-1e-4, 1e-4, 300).astype(np.float32)
    vpr = rng.uniform(-1e-5, 1e-5, 300).astype(np.float32)
    idf = np.full(300, 3e4, np.float32)
    h = m3d.qlg_bot_profile(a, q, vpr, idf)
    th = ops.qlg_bot_profile(_dev(a), _dev(q), _dev(vpr), _dev(idf))
    np.testing.assert_array_equal(th.cpu().numpy(), h)


def test_stateq_op_matches_front_end(m3d, ops):
    import ctypes as C
    import torch
    from dispatch_b200 import stateq, synth
    atom, inp = synth.se_config("small", ncell=512)
    b = inp["b"].copy()
    res, lvl = stateq.stateq_update(atom, b, inp["nstar"], inp["totn"], inp["e_kT"], inp["gamma_ij"],
                                    inp["gamma_ji"], temp=inp["temp"], ne=inp["ne"])
    st, keep = stateq.make_atom(atom)
    T, NE = _dev(np.asarray(inp["temp"], np.float64)), _dev(np.asarray(inp["ne"], np.float64))
    cells, keep2 = stateq._cells(T, NE, None, None, None, None)
    tb = _dev(inp["b"])
    tl = torch.zeros(st.nlevel, dtype=torch.float64)
    out = ops.stateq_update(C.addressof(st), C.addressof(cells), 0, [1e2, 1.0, 1e-30, 0.0, 1e7, 1.0], tb,
                            _dev(inp["nstar"]), _dev(inp["totn"]), _dev(inp["e_kT"]), _dev(inp["gamma_ij"]),
                            _dev(inp["gamma_ji"]), None, tl)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(tb.cpu().numpy(), b)
    assert float(out[0]) == res["maxerr"]
    np.testing.assert_array_equal(tl.numpy(), lvl)

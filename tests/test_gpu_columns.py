"""The batched 1.5D ALI through the library's column plan (dispatch_b200.ali.AliColumns)
against the oracle's composition (oracle/ali.py: run_columns), on seeded columns of
uneven depth, a model atom split over two frequency windows and abundance variants.

A sweep is bit-exact: the same FP32 kernels and the long-characteristics solver along
each column, which the oracle runs as one 1-column slab per column.  The sweep
replayed from the CUDA graph equals the directly launched one bit for bit.  Over
several iterations the departure coefficients carry the device's exp/log in the
collision rates (1e-10 per update) and stay within 1e-7 of the oracle's.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(sums=False, variants=(0.0, 0.2)):
    from dispatch_b200 import ali, synth
    cols, atom, wins, mu, wmu = ali.column_problem(variants=variants)
    if sums:
        nrad = len(atom["ti"])
        s = (np.arange(atom["nline"]) % 2 == 0).astype(np.uint8)
        wins = [synth.atom_window(atom, seed=3, transitions=list(range(k, nrad, 2)), sums=s) for k in range(2)]
    return cols, atom, wins, mu, wmu


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("sums", [False, True])
def test_column_sweep_bit_exact(m3d, oracle, sums, fused):
    """The fused column sweep (one kernel per window and hemisphere) and the
    per-point kernels both equal the oracle bit for bit."""
    from dispatch_b200 import ali
    from oracle import ali as oali
    cols, atom, wins, mu, wmu = _problem(sums)
    S = oali.setup_columns(cols, atom, wins, mu, wmu)
    oali.sweep_columns(S)
    A = ali.AliColumns(cols, atom, wins, mu, wmu, use_graph=False, fused=fused)
    assert A.shape["fused_windows"] == (len(wins) if fused else 0)
    A.sweep()
    np.testing.assert_array_equal(A.gamma_ij.cpu().numpy(), S["gamma_ij"])
    np.testing.assert_array_equal(A.gamma_ji.cpu().numpy(), S["gamma_ji"])
    J, P = A.fields()
    np.testing.assert_array_equal(J.cpu().numpy(), S["J"])
    np.testing.assert_array_equal(P.cpu().numpy(), S["PsiJ"])
    np.testing.assert_array_equal(A.wphi.cpu().numpy(), S["wphi"])
    assert np.abs(S["gamma_ij"]).max() > 0
    if sums:
        assert S["wphi"].max() > 0
    A.close()


def _overlap_problem():
    """Columns with an atom whose line windows overlap: one window where up to 3
    lines share a frequency (fused) and one where up to 9 do (more than the fused
    kernel keeps in registers: the per-point kernels)."""
    from dispatch_b200 import ali, synth
    cols, _, _, mu, wmu = ali.column_problem(variants=(0.0, 0.2))
    atom = synth.model_atom(3, nbound=8, nline=20)
    nrad = len(atom["ti"])
    wins = [synth.atom_window(atom, seed=3, qmax_doppler=5000.0, transitions=list(range(0, nrad, 2))),
            synth.atom_window(atom, seed=3, qmax_doppler=60000.0, transitions=list(range(1, nrad, 2)))]
    nper = []
    for w in wins:
        c = np.zeros(w["nf"], int)
        for b, r in zip(w["line_blue"], w["line_red"]):
            c[b:r + 1] += 1
        nper.append(int(c.max()))
    assert 1 < nper[0] <= 4 < nper[1]
    return cols, atom, wins, mu, wmu


def test_column_sweep_overlapping_lines_bit_exact(m3d, oracle):
    """Several lines on one frequency: the split tracking across lines and the rate
    rows of each line in the fused kernel, and a window past its limit swept by the
    per-point kernels within the same plan, all equal to the oracle bit for bit."""
    from dispatch_b200 import ali
    from oracle import ali as oali
    cols, atom, wins, mu, wmu = _overlap_problem()
    S = oali.setup_columns(cols, atom, wins, mu, wmu)
    oali.sweep_columns(S)
    A = ali.AliColumns(cols, atom, wins, mu, wmu, use_graph=False)
    assert A.shape["fused_windows"] == 1
    A.sweep()
    np.testing.assert_array_equal(A.gamma_ij.cpu().numpy(), S["gamma_ij"])
    np.testing.assert_array_equal(A.gamma_ji.cpu().numpy(), S["gamma_ji"])
    J, P = A.fields()
    np.testing.assert_array_equal(J.cpu().numpy(), S["J"])
    np.testing.assert_array_equal(P.cpu().numpy(), S["PsiJ"])
    A.close()


@pytest.mark.parametrize("precond", [True, False])
@pytest.mark.parametrize("bottom", ["pchip", "zero"])
def test_fused_equals_per_point(m3d, precond, bottom):
    """The fused sweep and the per-point kernels give the same rates and fields bit
    for bit with and without preconditioning and with either bottom ghost, over
    two iterations (the update in between) and a third sweep, from the CUDA graph."""
    from dispatch_b200 import BND_PCHIP, BND_ZERO, ali
    cols, atom, wins, mu, wmu = _overlap_problem()
    p = ali.AliParams(preconditioning=precond, bottom=BND_PCHIP if bottom == "pchip" else BND_ZERO, convlim=1e-9)
    out = []
    for fused in (True, False):
        A = ali.AliColumns(cols, atom, wins, mu, wmu, params=p, fused=fused)
        A.run(2)
        A.sweep()
        J, P = A.fields()
        out.append((A.b.cpu().numpy(), A.gamma_ij.cpu().numpy(), A.gamma_ji.cpu().numpy(), J.cpu().numpy(),
                    P.cpu().numpy(), [h["maxerr"] for h in A.history]))
        A.close()
    for a, b in zip(out[0][:5], out[1][:5]):
        np.testing.assert_array_equal(a, b)
    assert out[0][5] == out[1][5]
    assert np.abs(out[0][1]).max() > 0 and np.abs(out[0][0] - 1.0).max() > 0.01


def test_column_graph_replay_equals_launches(m3d):
    from dispatch_b200 import ali
    cols, atom, wins, mu, wmu = _problem()
    runs = []
    for graph in (False, True):
        A = ali.AliColumns(cols, atom, wins, mu, wmu, use_graph=graph, params=ali.AliParams(convlim=1e-9))
        A.run(4)
        runs.append((A.b.cpu().numpy(), [h["maxerr"] for h in A.history]))
        A.close()
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_column_iterations_match_oracle(m3d, oracle):
    from dispatch_b200 import ali
    from oracle import ali as oali
    cols, atom, wins, mu, wmu = _problem(variants=(0.0, 0.2, -0.2))
    hist_o, S = oali.run_columns(cols, atom, wins, mu, wmu, maxiter=6, convlim=1e-6)
    A = ali.AliColumns(cols, atom, wins, mu, wmu, params=ali.AliParams(convlim=1e-6))
    hist_g = A.run(6)
    assert len(hist_g) == len(hist_o) == 6
    for g, o in zip(hist_g, hist_o):
        assert g["maxerr"] == pytest.approx(o["maxerr"], rel=1e-7)
    np.testing.assert_allclose(A.b.cpu().numpy(), S["b"], rtol=1e-7)
    assert np.abs(S["b"] - 1.0).max() > 0.05
    # the variants differ only in abundance: their columns do not share populations
    nc1 = int(cols["col_off"][len(cols["col_off"]) // 3])
    assert not np.allclose(S["b"][:, :nc1], S["b"][:, nc1:2 * nc1])
    assert A.solver_block in (64, 128, 256, 512)
    assert A.shape["fused_windows"] == len(wins) and A.shape["zchunk"] in (4, 8, 16)
    A.close()


def test_column_plan_rejects_bad_input(m3d):
    import torch
    from dispatch_b200 import ali
    cols, atom, wins, mu, wmu = _problem(variants=(0.0,))
    bad = dict(cols)
    off = cols["col_off"].copy()
    off[1] = off[0] + 1                      # a column of one cell
    bad["col_off"] = off
    with pytest.raises(m3d.M3DError, match="fewer than 2 cells"):
        ali.AliColumns(bad, atom, wins, mu, wmu)
    with pytest.raises(m3d.M3DError, match="mirrored"):
        ali.AliColumns(cols, atom, wins, mu[::-1].copy(), wmu)
    torch.cuda.synchronize()
    assert m3d.lib().m3d_col_plan_destroy(C.c_void_p()) == 0


def test_windows_shared_over_ranks_equal_one_plan(m3d):
    """The frequency-sharded iteration on one GPU: two plans each holding every
    other window (what two ranks hold), their rates summed as the exchange sums
    them, equal the plan of all windows bit for bit (every transition sits in one
    window), and so does the update that follows."""
    from dispatch_b200 import ali
    cols, atom, wins, mu, wmu = _problem(sums=True)
    wins = wins + [w for w in _problem()[2]]      # four windows
    full = ali.AliColumns(cols, atom, wins, mu, wmu, use_graph=False)
    part = [ali.AliColumns(cols, atom, wins, mu, wmu, use_graph=False, windows=list(range(r, len(wins), 2)))
            for r in range(2)]
    for A in [full] + part:
        A.sweep()
    for name in ("gamma_ij", "gamma_ji", "wphi"):
        s = getattr(part[0], name) + getattr(part[1], name)
        np.testing.assert_array_equal(s.cpu().numpy(), getattr(full, name).cpu().numpy())
        getattr(part[0], name).copy_(s)
    for A in (full, part[0]):
        A.iter = 1
        A.update()
    np.testing.assert_array_equal(part[0].b.cpu().numpy(), full.b.cpu().numpy())
    for A in [full] + part:
        A.close()


def test_process_group_of_one_runs_the_exchange(m3d):
    """A one-rank NCCL group: the windows all stay on the rank and run() calls the
    exchange each iteration; the iterations equal those without a group."""
    import socket

    import torch
    import torch.distributed as dist
    from dispatch_b200 import ali
    cols, atom, wins, mu, wmu = _problem()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    from datetime import timedelta
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        A = ali.AliColumns(cols, atom, wins, mu, wmu, params=ali.AliParams(convlim=1e-9), group=dist.group.WORLD,
                           use_graph=False)
        A.run(3)
        B = ali.AliColumns(cols, atom, wins, mu, wmu, params=ali.AliParams(convlim=1e-9), use_graph=False)
        B.run(3)
        np.testing.assert_array_equal(A.b.cpu().numpy(), B.b.cpu().numpy())
        A.close()
        B.close()
    finally:
        dist.destroy_process_group()

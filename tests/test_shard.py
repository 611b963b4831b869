"""Window sharding across ranks: world-size-2 gloo processes on CPU."""
import os

import numpy as np
import pytest


def test_windows_partition():
    from dispatch_b200.shard import windows_for_rank
    for world in (1, 2, 3, 8):
        got = sorted(w for r in range(world) for w in windows_for_rank(r, world, 125))
        assert got == list(range(125))
    with pytest.raises(ValueError):
        windows_for_rank(2, 2, 10)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dispatch_b200.shard import gather_spectrum, max_over_ranks, windows_for_rank
        nwin, nf = 7, 4
        local = {w: np.arange(nf) + 100.0 * w for w in windows_for_rank(rank, world, nwin)}
        full = gather_spectrum(local, nwin, nf)
        t = max_over_ranks(10.0 + rank)
        q.put((rank, full.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    exp = (np.arange(4)[None, :] + 100.0 * np.arange(7)[:, None]).ravel()
    for rank, full, t in res:
        np.testing.assert_array_equal(full, exp)
        assert t == 11.0


def _rates_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dispatch_b200 import ali
        from dispatch_b200.shard import allreduce_rates, windows_for_rank
        from oracle import ali as oali
        cols, atom, wins, mu, wmu = ali.column_problem(variants=(0.0,))
        mine = [wins[w] for w in windows_for_rank(rank, world, len(wins))]
        S = oali.setup_columns(cols, atom, mine, mu, wmu)
        oali.sweep_columns(S)
        gij, gji = torch.from_numpy(S["gamma_ij"].copy()), torch.from_numpy(S["gamma_ji"].copy())
        wphi = torch.from_numpy(S["wphi"].copy())
        allreduce_rates(gij, gji, wphi)
        q.put((rank, gij.numpy(), gji.numpy(), wphi.numpy()))
    finally:
        dist.destroy_process_group()


def test_rates_summed_over_two_gloo_ranks_equal_one_rank():
    """Two ranks each sweep half of the atom's windows (the oracle's composition
    stands in for the device sweep on CPU) and sum their rates with the NLTE
    exchange: every transition sits in one window, so the sums equal the single
    sweep over all windows bit for bit."""
    import multiprocessing as mp
    import socket
    from dispatch_b200 import ali
    from oracle import ali as oali
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rates_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cols, atom, wins, mu, wmu = ali.column_problem(variants=(0.0,))
    S = oali.setup_columns(cols, atom, wins, mu, wmu)
    oali.sweep_columns(S)
    for rank, gij, gji, wphi in res:
        np.testing.assert_array_equal(gij, S["gamma_ij"])
        np.testing.assert_array_equal(gji, S["gamma_ji"])
        np.testing.assert_array_equal(wphi, S["wphi"])
    assert np.abs(S["gamma_ij"]).max() > 0


def _chunk_windows():
    """The column problem's atom split into three contiguous wavelength chunks, so
    that continua span all three windows."""
    from dispatch_b200 import ali, synth
    cols, atom, _, mu, wmu = ali.column_problem(variants=(0.0,))
    lam = synth.atom_window(atom, nper=25, seed=3)["lam"]
    cuts = np.quantile(lam, [0.0, 1.0 / 3.0, 2.0 / 3.0, 1.0])
    cuts[-1] = lam.max() * 1.001
    wins = [synth.atom_window(atom, nper=25, seed=3, lam_range=(cuts[i], cuts[i + 1])) for i in range(3)]
    return cols, atom, wins, mu, wmu


def _chunk_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dispatch_b200.shard import allreduce_rates, windows_for_rank
        from oracle import ali as oali
        cols, atom, wins, mu, wmu = _chunk_windows()
        mine = [wins[w] for w in windows_for_rank(rank, world, len(wins))]
        S = oali.setup_columns(cols, atom, mine, mu, wmu)
        oali.sweep_columns(S)
        gij, gji = torch.from_numpy(S["gamma_ij"].copy()), torch.from_numpy(S["gamma_ji"].copy())
        allreduce_rates(gij, gji)
        q.put((rank, gij.numpy(), gji.numpy()))
    finally:
        dist.destroy_process_group()


def test_continuum_across_windows_on_two_gloo_ranks():
    """Three contiguous wavelength windows, continua spanning all of them; rank 0
    sweeps windows 0 and 2, rank 1 window 1, and the exchange sums their rates.  One
    rank sums (w0 + w1) + w2, two ranks (w0 + w2) + w1: a transition confined to one
    window is summed exactly, one spanning windows differs by the float32
    reassociation, at most 2 ulp (relative 2.4e-7)."""
    import multiprocessing as mp
    import socket
    from oracle import ali as oali
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_chunk_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cols, atom, wins, mu, wmu = _chunk_windows()
    S = oali.setup_columns(cols, atom, wins, mu, wmu)
    oali.sweep_columns(S)
    spans = {}
    for w in wins:
        for k in list(w["line_ntrans"]) + list(w["cont_ntrans"]):
            spans[int(k)] = spans.get(int(k), 0) + 1
    multi = [k for k, n in spans.items() if n > 1]
    single = [k for k, n in spans.items() if n == 1]
    assert any(k >= atom["nline"] for k in multi)          # a continuum spans windows
    for rank, gij, gji in res:
        for g, ref in ((gij, S["gamma_ij"]), (gji, S["gamma_ji"])):
            np.testing.assert_array_equal(g[single], ref[single])
            np.testing.assert_allclose(g[multi], ref[multi], rtol=2.4e-7, atol=0)

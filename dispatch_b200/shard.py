"""Frequency windows across ranks (one process per GPU).

The reference splits the spectrum into n_windows frequency windows whose
opacities and sweeps are independent for all rays (E/SRC/ray_patch_mod.f90:97-127).
A rank takes every world-th window.  In LTE the spectra of the windows a rank
computed are gathered to every rank only for output, and the step time reported
is the maximum over ranks.  In an NLTE iteration the radiative rates are sums over
all windows: each rank sums its own windows' rates, one all-reduce (sum) per
iteration forms the totals on every rank (and once the profile integrals of the
first sweep), and every rank then takes the same statistical-equilibrium update.
"""
from __future__ import annotations

import numpy as np


def windows_for_rank(rank: int, world: int, nwin: int) -> list[int]:
    """Round-robin: rank r takes windows r, r + world, r + 2 world, ..."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world {world}")
    return list(range(rank, nwin, world))


def gather_spectrum(local: dict[int, np.ndarray], nwin: int, nf: int) -> np.ndarray:
    """Assemble the full spectrum (nwin * nf) from every rank's {window: flux(nf)}
    with torch.distributed (any backend); ranks must call it together."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    rank = dist.get_rank()
    mine = windows_for_rank(rank, world, nwin)
    if sorted(local) != mine:
        raise ValueError(f"rank {rank} holds windows {sorted(local)}, expected {mine}")
    nmax = len(windows_for_rank(0, world, nwin))
    buf = torch.zeros((nmax, nf), dtype=torch.float64)
    for i, w in enumerate(mine):
        buf[i] = torch.as_tensor(np.asarray(local[w], np.float64))
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.zeros((nwin, nf))
    for r in range(world):
        for i, w in enumerate(windows_for_rank(r, world, nwin)):
            out[w] = parts[r][i].numpy()
    return out.ravel()


def max_over_ranks(ms: float) -> float:
    """The slowest rank's time, the figure a weak-scaling step reports."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_rates(gamma_ij, gamma_ji, wphi=None, group=None) -> None:
    """The NLTE exchange of one ALI iteration: gamma_ij and gamma_ji (nrad, ncell),
    and the profile integrals wphi of the first sweep when given, summed over the
    ranks in place (torch.distributed; NCCL on the GPUs, gloo on CPU).  The sum
    groups the windows by rank, so against one rank summing every window in order
    the rates differ by float32 reassociation only."""
    import torch.distributed as dist

    for t in (gamma_ij, gamma_ji, wphi):
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

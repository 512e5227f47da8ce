"""Multi-GPU target sharding: one process per GPU, no data-path collective.

Kriging targets are independent (each solve reads only the observations and
its own target), so N GPUs split the targets into contiguous slabs, each rank
solves its slab with its own handle, and the only communication is the
optional gather of the results at the end.  Observations and their search
grid are replicated per rank (a few MB).

The helpers take any object with the ``Kriging`` setter/solve/get_results
interface, so the same code path runs the GPU class in production and a CPU
stand-in in host-only tests.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np


def target_slab(ntarget: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [lo, hi) slab of rank ``rank``: sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(int(ntarget), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def solve_slab(make_solver: Callable[[], object], grid: np.ndarray, rank: int, world: int,
               grid_drift: Optional[np.ndarray] = None, **set_grid_kw):
    """Configure a solver, give it this rank's slab of ``grid`` and solve.

    ``make_solver()`` returns an object with observations, variogram and search
    already set.  Returns ``(lo, hi, estimate, variance)`` of the slab.
    """
    lo, hi = target_slab(len(grid), rank, world)
    k = make_solver()
    kw = {key: (None if val is None else np.asarray(val)[lo:hi]) for key, val in set_grid_kw.items()}
    k.set_grid(np.asarray(grid)[lo:hi], **kw)
    if grid_drift is not None:
        k.set_grid_drift(np.asarray(grid_drift)[lo:hi])
    k.solve()
    est, var = k.get_results()
    return lo, hi, np.asarray(est), np.asarray(var)


def gather_slabs(lo: int, hi: int, est: np.ndarray, var: np.ndarray, ntarget: int, group=None):
    """Assemble every rank's slab on every rank (torch.distributed all_gather_object).

    Only the finished results cross between ranks; the solves never wait on
    one another.
    """
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, (lo, hi, est, var), group=group)
    e_all = np.empty((ntarget,) + est.shape[1:], dtype=est.dtype)
    v_all = np.empty((ntarget,) + var.shape[1:], dtype=var.dtype)
    for plo, phi, pe, pv in parts:
        e_all[plo:phi] = pe
        v_all[plo:phi] = pv
    return e_all, v_all

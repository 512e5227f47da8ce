"""Host-side multi-rank sharding, world size 2 over gloo on CPU.

Each rank solves its contiguous slab of the targets with the CPU oracle as
stand-in solver (the GPU class has the same interface); the gathered result
must equal one single-process solve of all targets, bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import bench_workloads as bw
from krigekit_b200.shard import gather_slabs, solve_slab, target_slab


def test_target_slab_partition():
    for n in (0, 1, 7, 10, 1001):
        for world in (1, 2, 3, 8):
            slabs = [target_slab(n, r, world) for r in range(world)]
            assert slabs[0][0] == 0 and slabs[-1][1] == n
            for (a, b), (c, _) in zip(slabs, slabs[1:]):
                assert b == c
            sizes = [b - a for a, b in slabs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        target_slab(10, 2, 2)


def _workload():
    return bw.config1(grid_n=13, nobs=400)


def _make_oracle():
    from oracle.oracle import OracleKriging
    w = _workload()
    return bw.apply(OracleKriging(ndim=2, nvar=1, nmin=4), w, set_grid=False)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grid = _workload()["grid"]
        lo, hi, e, v = solve_slab(_make_oracle, grid, rank, world)
        e_all, v_all = gather_slabs(lo, hi, e, v, len(grid))
        np.save(os.path.join(out_dir, f"est{rank}.npy"), e_all)
        np.save(os.path.join(out_dir, f"var{rank}.npy"), v_all)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_matches_single_process(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    k = _make_oracle()
    k.set_grid(_workload()["grid"])
    k.solve()
    e_ref, v_ref = k.get_results()
    for r in range(world):
        np.testing.assert_array_equal(np.load(tmp_path / f"est{r}.npy"), e_ref)
        np.testing.assert_array_equal(np.load(tmp_path / f"var{r}.npy"), v_ref)

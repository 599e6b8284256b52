"""The z-slab exchange plan on CPU: world sizes 1-4 as gloo ranks.

Each rank holds a population array [19, L, ny, nx] (L = its planes + 2 ghosts)
filled with values that name (rank, slot, plane, cell).  After phase 0 every
ghost plane must hold, in its 5 crossing slots, the neighbour's boundary plane;
after phase 1 every boundary plane must hold, in those slots, what the
neighbour's ghost plane held.  All other slots stay untouched.
"""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from myfluidsimulation_b200.slabs import STAT_KEYS, exchange, exchange_plan, reduce_stats, slab_bounds, with_ghosts

UP = [q for q in range(19) if q in (5, 11, 12, 15, 16)]     # c_z = +1
DOWN = [q for q in range(19) if q in (6, 13, 14, 17, 18)]   # c_z = -1


def _fill(rank, L, ny, nx):
    a = np.zeros((19, L, ny, nx), np.float32)
    for q in range(19):
        for pl in range(L):
            a[q, pl] = 1e6 * rank + 1e4 * q + 100 * pl + np.arange(ny * nx).reshape(ny, nx) % 97
    return a


def _worker(rank, world, port, nz, ny, nx, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        z0, z1 = slab_bounds(nz, world)[rank]
        L = z1 - z0 + 2
        a = torch.from_numpy(_fill(rank, L, ny, nx))
        planes = {"ghost_lo": 0, "first": 1, "last": L - 2, "ghost_hi": L - 1}
        views = {(n, cz): [a[q, pl].view(-1) for q in (UP if cz > 0 else DOWN)] for n, pl in planes.items()
                 for cz in (1, -1)}
        exchange(views, 0, rank, world, dist)
        after0 = a.numpy().copy()
        exchange(views, 1, rank, world, dist)
        out[rank] = (after0, a.numpy().copy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_exchange_moves_exactly_the_crossing_slots(world):
    nz, ny, nx = 11, 3, 4
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = 29600 + world
    procs = [ctx.Process(target=_worker, args=(r, world, port, nz, ny, nx, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    bounds = slab_bounds(nz, world)
    for r in range(world):
        lo, hi = (r - 1) % world, (r + 1) % world
        L = bounds[r][1] - bounds[r][0] + 2
        Llo = bounds[lo][1] - bounds[lo][0] + 2
        a0 = _fill(r, L, ny, nx)
        after0, after1 = out[r]
        want0 = a0.copy()
        want0[DOWN, 0] = _fill(lo, Llo, ny, nx)[DOWN, Llo - 2]     # lower's last own plane
        want0[UP, L - 1] = _fill(hi, bounds[hi][1] - bounds[hi][0] + 2, ny, nx)[UP, 1]
        np.testing.assert_array_equal(after0, want0)
        # phase 1: the upper neighbour's ghost_lo (after its phase 0) comes back into my last plane
        Lhi = bounds[hi][1] - bounds[hi][0] + 2
        want1 = want0.copy()
        hi_after0 = out[hi][0]
        lo_after0 = out[lo][0]
        want1[DOWN, L - 2] = hi_after0[DOWN, 0]
        want1[UP, 1] = lo_after0[UP, Llo - 1]
        np.testing.assert_array_equal(after1, want1)


def test_plan_pairs_and_bounds():
    assert slab_bounds(10, 3) == [(0, 3), (3, 6), (6, 10)]
    for world in (2, 3, 5):
        for phase in (0, 1):
            sends = {(r, p, pl, cz) for r in range(world) for k, p, pl, cz in exchange_plan(phase, r, world)
                     if k == "send"}
            recvs = {(p, r) for r in range(world) for k, p, pl, cz in exchange_plan(phase, r, world) if k == "recv"}
            assert {(r, p) for r, p, _, _ in sends} == recvs
    a = np.arange(5 * 2).reshape(5, 2)
    np.testing.assert_array_equal(with_ghosts(a, 0, 2), a[[4, 0, 1, 2]])
    np.testing.assert_array_equal(with_ghosts(a, 3, 5), a[[2, 3, 4, 0]])


def _stats_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = {k: (rank + 1) * 10.0 ** i + 0.125 * i for i, k in enumerate(STAT_KEYS)}
        out[rank] = reduce_stats(local, 1000, dist)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_reduce_stats_sums_over_ranks(world):
    """The slabs' FP64 statistics all-reduce as gloo ranks: every rank gets the
    sum of all ranks' values, and the mean energy over the whole grid."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = 29650 + world
    procs = [ctx.Process(target=_stats_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        got = out[r]
        for i, k in enumerate(STAT_KEYS):
            want = sum((q + 1) * 10.0 ** i + 0.125 * i for q in range(world))
            assert got[k] == want
        assert got["ke_mean"] == got["ke_sum"] / 1000

"""Scene-parallel placement of the batched and served forms over ranks (CPU, gloo).

Every rank computes the same assignment on its own (no data-path collective); the union of
the ranks' shares is every scene exactly once, the largest share exceeds the mean by at most
one scene, and the benchmark's only collective (the max / sum over ranks of a rank's time
or work) gives every rank the same answer.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from vxl_sph import placement


def test_assign_single_rank_is_everything():
    sizes = [5, 1, 9, 3]
    assert placement.assign_scenes(sizes, 1) == [[0, 1, 2, 3]]


def test_assign_balances_and_covers():
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(3))
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(4096), np.log(262144), 256))]
    for world in (2, 3, 4, 8):
        parts = placement.assign_scenes(sizes, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert placement.assign_scenes(sizes, world) == parts  # deterministic


def test_assign_more_ranks_than_scenes():
    parts = placement.assign_scenes([7, 3], 4)
    assert parts == [[0], [1], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = placement.assign_scenes(sizes, world)[rank]
        work = float(sum(sizes[i] for i in mine))
        t = float(rank + 1) * 1.5  # stand-in for this rank's measured time
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        q.put((rank, shares, placement.max_over_ranks(t, dist), placement.sum_over_ranks(work, dist)))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_placement_and_reductions():
    sizes = [262144, 4096, 50000, 120000, 9000, 70000, 33000]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = placement.assign_scenes(sizes, world)
    for rank, shares, tmax, wsum in res:
        assert shares == expect
        assert tmax == pytest.approx(1.5 * world)
        assert wsum == pytest.approx(float(sum(sizes)))

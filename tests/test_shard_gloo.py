"""Lane sharding over two ranks (gloo on CPU, world_size 2): each rank
solves its block of sweep points with the CPU oracle, the blocks gathered in
rank order equal the single-process batch bitwise, and the run reductions
give the slowest rank's time and the total point count."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from espice_b200 import decks, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        fr, slots, values = decks.grid_diodes(points=67)
        lo, hi = shard.block(len(values), rank, world)
        x, it, cv = oracle.dc_points(fr, slots, values[lo:hi], warm=np.zeros(fr.n))
        rows = np.concatenate([x, it[:, None].astype(np.float64), cv[:, None].astype(np.float64)], axis=1)
        full = shard.gather_rows(rows, len(values))
        secs, count = shard.reduce_run(0.5 + rank, int(cv.sum()))
        if rank == 0:
            q.put((full, secs, count))
    finally:
        dist.destroy_process_group()


def test_blocks_cover_every_lane_once():
    for n in (0, 1, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                lo, hi = shard.block(n, r, world)
                got.extend(range(lo, hi))
            assert got == list(range(n))


def test_two_ranks_match_one_process():
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, secs, count = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fr, slots, values = decks.grid_diodes(points=67)
    x, it, cv = oracle.dc_points(fr, slots, values, warm=np.zeros(fr.n))
    assert np.array_equal(full[:, :fr.n].view(np.uint64), x.view(np.uint64))
    assert np.array_equal(full[:, fr.n].astype(np.uint32), it)
    assert secs == 1.5
    assert count == int(cv.sum())

"""Lane sharding across ranks (one process per GPU). Sweep points and
Monte-Carlo samples are independent, so a batch splits into disjoint
contiguous lane blocks with the topology replicated on every rank; nothing
is exchanged while the lanes solve. After a run the ranks agree on the
slowest rank's time and the total count (max and sum reductions), and the
results can be gathered to rank 0."""

from __future__ import annotations


def block(n, rank, world):
    """The contiguous lane block [lo, hi) of `rank` among `world` ranks."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def reduce_run(seconds, count):
    """(max seconds over ranks, sum of counts) on the default process group
    (a single process returns its own values)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds), int(count)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    c = torch.tensor([float(count)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(c.item())


def gather_rows(rows, n_total):
    """Every rank's row block (numpy [rows][k], in rank order) assembled on
    every rank into [n_total][k]."""
    import numpy as np
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return rows
    world = dist.get_world_size()
    k = rows.shape[1]
    width = max(block(n_total, r, world)[1] - block(n_total, r, world)[0] for r in range(world))
    pad = np.zeros((width, k), rows.dtype)
    pad[:rows.shape[0]] = rows
    t = torch.from_numpy(pad)
    out = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(out, t)
    parts = []
    for r in range(world):
        lo, hi = block(n_total, r, world)
        parts.append(out[r].numpy()[:hi - lo])
    return np.concatenate(parts)

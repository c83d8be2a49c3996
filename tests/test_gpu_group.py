"""Uneven batching and the lanes-per-CTA autotuner (B200).

Three circuits of different sizes and lane counts solved in one launch give
each lane bitwise the result of its own context's launch (the same per-lane
solve on the same tape); the autotuner's choice of lanes per CTA changes
timing only, never a result bit.
"""

import numpy as np
import pytest

from espice_b200 import decks, lanes

pytestmark = pytest.mark.gpu


def _case(rows, cols, n_diodes, points, seed):
    fr, slots, values = decks.grid_diodes(seed=seed, rows=rows, cols=cols, n_diodes=n_diodes, points=points)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    return fr, ctx


def test_group_launch_matches_single_launches():
    import torch
    cases = [_case(4, 4, 3, 37, 1), _case(8, 8, 16, 256, 2), _case(10, 12, 20, 100, 3)]
    opts = lanes.newton_opts()
    singles = []
    for fr, ctx in cases:
        x, it, st, _ = ctx.solve(x0=np.zeros(fr.n), opts=opts)
        singles.append((x, it, st))
    bufs = []
    for fr, ctx in cases:
        bufs.append((torch.zeros((ctx.n_lanes, fr.n), dtype=torch.float64, device="cuda"),
                     torch.zeros(ctx.n_lanes, dtype=torch.int32, device="cuda"),
                     torch.zeros(ctx.n_lanes, dtype=torch.int32, device="cuda")))
    torch.cuda.synchronize()
    stats = lanes.group_solve_device([c for _, c in cases], [b[0].data_ptr() for b in bufs],
                                     [b[1].data_ptr() for b in bufs], [b[2].data_ptr() for b in bufs], opts=opts)
    torch.cuda.synchronize()
    for (x, it, st), (dx, di, ds), s, (fr, ctx) in zip(singles, bufs, stats, cases):
        assert np.array_equal(dx.cpu().numpy().view(np.uint64), x.view(np.uint64))
        assert np.array_equal(di.cpu().numpy().astype(np.uint32), it)
        assert np.array_equal(ds.cpu().numpy().astype(np.uint32), st)
        assert s["lanes"] == ctx.n_lanes and s["converged"] == int((st == lanes.LANE_CONVERGED).sum())
    for _, ctx in cases:
        ctx.close()


def test_autotune_keeps_results():
    fr, ctx = _case(8, 8, 16, 512, 4)
    x0 = np.zeros(fr.n)
    x1, it1, st1, _ = ctx.solve(x0=x0)
    best = ctx.autotune(x0=x0)
    assert best in (1, 2, 4, 8)
    x2, it2, st2, _ = ctx.solve(x0=x0)
    assert np.array_equal(x1.view(np.uint64), x2.view(np.uint64))
    assert np.array_equal(it1, it2) and np.array_equal(st1, st2)
    ctx.close()

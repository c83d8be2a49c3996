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


@pytest.mark.parametrize("precision", [lanes.PREC_FP64, lanes.PREC_MIXED])
def test_block_group_uneven_batch_against_oracle(precision):
    """The uneven batch on the block lanes: the eight mesh-with-gates
    topologies (50 to 2,000 unknowns), six supply values each, in one launch
    (work items largest topology first; the two largest keep their working
    set in global memory). FP64: every lane bitwise the oracle, the same
    iteration counts. Mixed: the oracle's convergence, values within 1e-9
    relative or 1e-12 absolute."""
    import torch
    import parity
    from oracle import oracle
    vals = np.linspace(0.8, 1.8, 6).reshape(-1, 1)
    ctxs, bufs, decks_ = [], [], []
    for size in decks.MESH_GATES_SIZES:
        fr, slots = decks.mesh_gates(size)
        c = lanes.DcLanes(fr)
        c.set_mode(precision=precision, path=lanes.PATH_BLOCK)
        c.set_lanes(slots, vals)
        ctxs.append(c)
        decks_.append((fr, slots))
        bufs.append((torch.zeros((len(vals), fr.n), dtype=torch.float64, device="cuda"),
                     torch.zeros(len(vals), dtype=torch.int32, device="cuda"),
                     torch.zeros(len(vals), dtype=torch.int32, device="cuda")))
    torch.cuda.synchronize()
    stats = lanes.group_solve_device(ctxs, [b[0].data_ptr() for b in bufs], [b[1].data_ptr() for b in bufs],
                                     [b[2].data_ptr() for b in bufs], cold=[True] * len(ctxs))
    torch.cuda.synchronize()
    for (fr, slots), b, s, c in zip(decks_, bufs, stats, ctxs):
        assert s["path"] == lanes.PATH_BLOCK
        x = b[0].cpu().numpy()
        it = b[1].cpu().numpy().astype(np.uint32)
        st = b[2].cpu().numpy().astype(np.uint32)
        xo, ito, cvo = oracle.dc_points(fr, slots, vals, warm=None)
        conv = st == lanes.LANE_CONVERGED
        if precision == lanes.PREC_FP64:
            assert parity.assert_dc_parity(fr, slots, vals, None, oracle.newton_opts(), x, it, conv, xo, ito, cvo,
                                           f"group n={fr.n}") == 1.0
        else:
            assert np.array_equal(conv, cvo.astype(bool))
            assert parity.close(x[conv], xo[conv]).all(), float(np.max(np.abs(x[conv] - xo[conv])))
        c.close()

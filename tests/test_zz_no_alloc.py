"""The allocation-free DC entry point, esl_dc_solve_device_static, against
esl_dc_solve_device on the same lanes.

Both run the same fused kernel on the same lead pivot tape; only where the
per-lane Newton state lives differs (the library's fixed device array versus
the context's allocations), so the lanes agree: the same status and Newton
iteration count, x within the lane parity tolerance (1e-9 relative or 1e-12
absolute; equal bits are expected). Each case makes two static calls in a
row. Lanes that leave the lead tape are not served by the static entry: they
come back as ESL_LANE_NEED_SOLVE with the call refused.
"""

import numpy as np
import pytest

from espice_b200 import decks, lanes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-12


def _torch():
    import torch
    assert torch.cuda.is_available(), "a CUDA device is required"
    return torch


def _close(a, b):
    return np.abs(a - b) <= ATOL + RTOL * np.maximum(np.abs(a), np.abs(b))


def _buffers(torch, x0):
    d_x = torch.tensor(x0, dtype=torch.float64, device="cuda")
    d_it = torch.zeros(x0.shape[0], dtype=torch.int32, device="cuda")
    d_st = torch.zeros(x0.shape[0], dtype=torch.int32, device="cuda")
    return d_x, d_it, d_st


def _ptrs(bufs):
    return [b.data_ptr() for b in bufs]


def _host(torch, bufs):
    torch.cuda.synchronize()
    return bufs[0].cpu().numpy(), bufs[1].cpu().numpy(), bufs[2].cpu().numpy()


@pytest.mark.parametrize("cold", [False, True])
def test_static_entry_matches_device_entry(cold):
    torch = _torch()
    fr, slots, values = decks.grid_diodes(seed=2, points=256)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    x0 = np.zeros((len(values), fr.n))
    ref_bufs = _buffers(torch, x0)
    torch.cuda.synchronize()
    stats = ctx.solve_device(*_ptrs(ref_bufs), cold=cold)
    xr, itr, str_ = _host(torch, ref_bufs)
    assert (str_ == lanes.LANE_CONVERGED).all()
    for call in range(2):
        bufs = _buffers(torch, x0)
        torch.cuda.synchronize()
        if stats["peeled"] == 0:
            assert ctx.solve_device_static(*_ptrs(bufs), cold=cold) == 0
        else:
            with pytest.raises(lanes.LaneError) as err:
                ctx.solve_device_static(*_ptrs(bufs), cold=cold)
            assert err.value.code == lanes.ESL_NOT_ELIGIBLE
        xs, its, sts = _host(torch, bufs)
        ok = sts != lanes.LANE_NEED_SOLVE
        assert (~ok).sum() <= stats["peeled"], f"call {call}"
        assert np.array_equal(sts[ok], str_[ok]), f"call {call}"
        assert np.array_equal(its[ok], itr[ok]), f"call {call}"
        assert _close(xs[ok], xr[ok]).all(), f"call {call}"
    ctx.close()


def test_static_entry_leaves_paused_lanes_to_the_caller():
    """A zener regulator swept into breakdown: some lanes leave the lead
    pivot tape. Twice in a row, the allocation-free call refuses with
    ESL_NOT_ELIGIBLE, reports exactly the lanes it left at
    ESL_LANE_NEED_SOLVE, and every other lane ends as the allocating entry
    point's does, bit for bit."""
    import golden_util as gu
    from netlist import Deck, sweep_values

    torch = _torch()
    g = gu.load("dc__bench_power_zener_reg")
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    values = np.array(sweep_values(an[2], an[3], an[4])).reshape(-1, 1)
    slots = [fr.slot(an[1], "dc")]
    opts = lanes.newton_opts(**deck.newton_opts())
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    x0 = np.zeros((len(values), fr.n))
    ref_bufs = _buffers(torch, x0)
    torch.cuda.synchronize()
    stats = ctx.solve_device(*_ptrs(ref_bufs), cold=True, opts=opts)
    xr, itr, str_ = _host(torch, ref_bufs)
    assert stats["peeled"] > 0, stats
    for call in range(2):
        bufs = _buffers(torch, x0)
        torch.cuda.synchronize()
        with pytest.raises(lanes.LaneError) as err:
            ctx.solve_device_static(*_ptrs(bufs), cold=True, opts=opts)
        assert err.value.code == lanes.ESL_NOT_ELIGIBLE
        xs, its, sts = _host(torch, bufs)
        paused = sts == lanes.LANE_NEED_SOLVE
        assert err.value.paused == int(paused.sum()) > 0, f"call {call}"
        assert int(paused.sum()) <= stats["peeled"], f"call {call}"
        ok = ~paused
        assert np.array_equal(sts[ok], str_[ok]), f"call {call}"
        assert np.array_equal(its[ok], itr[ok]), f"call {call}"
        assert np.array_equal(xs[ok].view(np.uint64), xr[ok].view(np.uint64)), f"call {call}"
    ctx.close()


def test_static_entry_needs_a_tape_first():
    torch = _torch()
    fr, slots, values = decks.grid_diodes(seed=3, points=32)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    bufs = _buffers(torch, np.zeros((32, fr.n)))
    torch.cuda.synchronize()
    with pytest.raises(lanes.LaneError) as err:
        ctx.solve_device_static(*_ptrs(bufs))
    assert err.value.code == lanes.ESL_NOT_ELIGIBLE
    assert "esl_dc_solve_device" in str(err.value)
    ctx.close()


def test_static_entry_refuses_lanes_beyond_its_scratch():
    """4096 lanes of this deck need about 20 MB of lane scratch, above the
    fixed 16 MiB: refused before any launch, the start points untouched."""
    torch = _torch()
    fr, slots, _ = decks.grid_diodes(seed=2, points=64)
    ctx = lanes.DcLanes(fr)
    values = np.linspace(0.0, 5.0, 4096).reshape(-1, 1)
    ctx.set_lanes(slots, values)
    x0 = np.full((4096, fr.n), 0.25)
    ref_bufs = _buffers(torch, x0)
    torch.cuda.synchronize()
    ctx.solve_device(*_ptrs(ref_bufs))
    bufs = _buffers(torch, x0)
    torch.cuda.synchronize()
    with pytest.raises(lanes.LaneError) as err:
        ctx.solve_device_static(*_ptrs(bufs))
    assert err.value.code == lanes.ESL_INVALID_ARGUMENT
    assert "lane scratch" in str(err.value)
    xs, _, _ = _host(torch, bufs)
    assert (xs == 0.25).all()
    ctx.close()

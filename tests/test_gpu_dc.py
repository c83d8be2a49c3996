"""GPU parity of the sweep-lane library against the CPU oracle (B200).

- The standalone lane refactor + solve kernel is bitwise the oracle's
  replay of the reference's column refactor and solve, peel verdicts
  included (lane_kernels.zig Bodies.refactor / solveNeg).
- The fused DC Newton kernel reproduces the oracle lane by lane: the same
  converged flag and exactly the same Newton iteration count on every lane
  (a flip fails the test and is reported with the oracle's gate inputs),
  and node voltages and branch currents within 1e-9 relative or 1e-12
  absolute on every lane. The device models and the oracle share one exp,
  log and pow (esl_math.h), so the synthetic decks' lanes are checked
  bitwise too.
- Golden fixtures of the reference, solved as independent GPU lanes from a
  cold start, meet the reference's own per-column tolerances.
"""

import numpy as np
import pytest

import golden_util as gu
import parity
from espice_b200 import decks, lanes
from netlist import Deck, sweep_values
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-12


def _torch():
    import torch
    assert torch.cuda.is_available(), "a CUDA device is required"
    return torch


def _close(a, b):
    return np.abs(a - b) <= ATOL + RTOL * np.maximum(np.abs(a), np.abs(b))


def _random_mna(n, seed, density=0.08):
    rng = np.random.default_rng(seed)
    cp = np.zeros(n + 1, np.uint32)
    ri, vals = [], []
    for j in range(n):
        rows = sorted({j} | {i for i in range(n) if i != j and rng.random() < density})
        off = {i: rng.uniform(-1, 1) for i in rows if i != j}
        zero = len(rows) > 1 and rng.random() < 0.15
        for i in rows:
            ri.append(i)
            vals.append(off[i] if i != j else (0.0 if zero else sum(abs(v) for v in off.values()) + 1.0))
        cp[j + 1] = len(ri)
    return cp, np.array(ri, np.uint32), np.array(vals)


@pytest.mark.parametrize("seed", range(6))
def test_lu_replay_kernel_bitwise(seed):
    torch = _torch()
    fr, slots, values = decks.grid_diodes(seed=seed + 1)
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(seed)
    lead = rng.uniform(0.5, 2.0, nnz) * np.where(rng.random(nnz) < 0.5, 1, -1)
    diag = np.array([np.searchsorted(ri[cp[j]:cp[j + 1]], j) + cp[j] for j in range(n)])
    lead[diag] += 8.0
    n_lanes = 97
    vals = np.stack([lead * rng.uniform(0.8, 1.2, nnz) for _ in range(n_lanes)])
    vals[0] = lead
    vals[5, diag[3]] = 0.0          # a lane whose pivot may die
    vals[7] *= 1e-9                 # a lane far from the lead's scale
    rhs = rng.normal(size=(n_lanes, n))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    ctx = lanes.DcLanes(fr)
    d_a = torch.tensor(vals, dtype=torch.float64, device="cuda")
    d_r = torch.tensor(rhs, dtype=torch.float64, device="cuda")
    d_dx = torch.zeros((n_lanes, n), dtype=torch.float64, device="cuda")
    d_bad = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_replay(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes)
    nu, nl, ntv = ctx.tape_size()
    d_tv = torch.zeros((n_lanes, ntv), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_replay(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes,
                  d_tv.data_ptr())
    torch.cuda.synchronize()
    bad = d_bad.cpu().numpy()
    assert np.array_equal(bad, ref["bad"])
    dx = d_dx.cpu().numpy()
    tv = d_tv.cpu().numpy()
    good = bad == 0
    assert good.sum() > n_lanes // 2
    assert np.array_equal(dx[good].view(np.uint64), ref["dx"][good].view(np.uint64))
    assert np.array_equal(tv[good, :nu].view(np.uint64), ref["ux"][good].view(np.uint64))
    assert np.array_equal(tv[good, nu + n:nu + n + nl].view(np.uint64), ref["lx"][good].view(np.uint64))
    ctx.close()


@pytest.mark.parametrize("deck,seed", [("grid", 0), ("grid", 3), ("ring", 1), ("ring", 2)])
def test_lu_lanes_kernel_bitwise(deck, seed):
    """The lane-interleaved kernel (one thread per lane, [entry][lane]
    planes) against the oracle's replay, bitwise, with pivot failures, on a
    lane count that is not a multiple of the warp or the CTA."""
    torch = _torch()
    fr = decks.grid_diodes(seed=seed + 1)[0] if deck == "grid" else decks.ring_oscillator(lanes=2)[0]
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(seed)
    lead = rng.uniform(0.5, 2.0, nnz) * np.where(rng.random(nnz) < 0.5, 1, -1)
    diag = np.array([np.searchsorted(ri[cp[j]:cp[j + 1]], j) + cp[j] for j in range(n)])
    lead[diag] += 8.0
    n_lanes = 333
    vals = np.stack([lead * rng.uniform(0.8, 1.2, nnz) for _ in range(n_lanes)])
    vals[0] = lead
    vals[5, diag[3]] = 0.0
    vals[7] *= 1e-9
    rhs = rng.normal(size=(n_lanes, n))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    ctx = lanes.DcLanes(fr)
    d_a = torch.tensor(vals.T.copy(), dtype=torch.float64, device="cuda")
    d_r = torch.tensor(rhs.T.copy(), dtype=torch.float64, device="cuda")
    d_dx = torch.zeros((n, n_lanes), dtype=torch.float64, device="cuda")
    d_bad = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_lanes(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes)
    nu, nl, ntv = ctx.tape_size()
    d_tv = torch.zeros((ntv, n_lanes), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_lanes(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes, d_tv.data_ptr())
    torch.cuda.synchronize()
    bad = d_bad.cpu().numpy()
    assert np.array_equal(bad, ref["bad"])
    dx = d_dx.cpu().numpy().T
    tv = d_tv.cpu().numpy().T
    good = bad == 0
    assert good.sum() > n_lanes // 2
    assert np.array_equal(dx[good].view(np.uint64), ref["dx"][good].view(np.uint64))
    assert np.array_equal(tv[good, :nu].view(np.uint64), ref["ux"][good].view(np.uint64))
    assert np.array_equal(tv[good, nu + n:nu + n + nl].view(np.uint64), ref["lx"][good].view(np.uint64))
    ctx.close()


@pytest.mark.parametrize("deck,seed", [("grid", 0), ("grid", 3), ("ring", 1), ("ring", 2)])
def test_lu_lanes_compiled_bitwise(deck, seed):
    """The tape compiled into code (esl_lu_lanes_compiled_device): bitwise
    the oracle's replay and the interpreted lane kernel, peel verdicts
    included, on a lane count that is not a multiple of the CTA."""
    torch = _torch()
    fr = decks.grid_diodes(seed=seed + 1)[0] if deck == "grid" else decks.ring_oscillator(lanes=2)[0]
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(seed)
    lead = rng.uniform(0.5, 2.0, nnz) * np.where(rng.random(nnz) < 0.5, 1, -1)
    diag = np.array([np.searchsorted(ri[cp[j]:cp[j + 1]], j) + cp[j] for j in range(n)])
    lead[diag] += 8.0
    n_lanes = 333
    vals = np.stack([lead * rng.uniform(0.8, 1.2, nnz) for _ in range(n_lanes)])
    vals[0] = lead
    vals[5, diag[3]] = 0.0
    vals[7] *= 1e-9
    rhs = rng.normal(size=(n_lanes, n))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    ctx = lanes.DcLanes(fr)
    d_a = torch.tensor(vals.T.copy(), dtype=torch.float64, device="cuda")
    d_r = torch.tensor(rhs.T.copy(), dtype=torch.float64, device="cuda")
    d_dx = torch.zeros((n, n_lanes), dtype=torch.float64, device="cuda")
    d_bad = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_lanes_compiled(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes)
    nu, nl, ntv = ctx.tape_size()
    d_tv = torch.zeros((ntv, n_lanes), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_lanes_compiled(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes,
                          d_tv.data_ptr())
    torch.cuda.synchronize()
    assert "registers" in ctx.lu_compiled_log()
    bad = d_bad.cpu().numpy()
    assert np.array_equal(bad, ref["bad"])
    dx = d_dx.cpu().numpy().T
    tv = d_tv.cpu().numpy().T
    good = bad == 0
    assert good.sum() > n_lanes // 2
    assert np.array_equal(dx[good].view(np.uint64), ref["dx"][good].view(np.uint64))
    assert np.array_equal(tv[good, :nu].view(np.uint64), ref["ux"][good].view(np.uint64))
    assert np.array_equal(tv[good, nu:nu + n].view(np.uint64), ref["udiag"][good].view(np.uint64))
    assert np.array_equal(tv[good, nu + n:nu + n + nl].view(np.uint64), ref["lx"][good].view(np.uint64))
    # the interpreted kernel on the same lanes: the same bits everywhere
    i_dx = torch.zeros_like(d_dx)
    i_tv = torch.zeros_like(d_tv)
    i_bad = torch.zeros_like(d_bad)
    ctx.lu_lanes(lead, d_a.data_ptr(), d_r.data_ptr(), i_dx.data_ptr(), i_bad.data_ptr(), n_lanes, i_tv.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(i_bad, d_bad)
    assert torch.equal(i_dx[:, torch.tensor(good, device="cuda")].view(torch.int64),
                       d_dx[:, torch.tensor(good, device="cuda")].view(torch.int64))
    ctx.close()


@pytest.mark.parametrize("deck,seed", [("grid", 0), ("ring", 1)])
def test_lu_lanes_mixed_compiled_matches_interpreted(deck, seed):
    """The mixed form compiled into code against the interpreted mixed
    kernel on the same lanes: the same peel verdicts and correction counts,
    dx within 1e-12 (the FP32 ops and the FP64 refinement run in the same
    per-value order)."""
    torch = _torch()
    fr = decks.grid_diodes(seed=seed + 1)[0] if deck == "grid" else decks.ring_oscillator(lanes=2)[0]
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(seed)
    lead = rng.uniform(0.5, 2.0, nnz) * np.where(rng.random(nnz) < 0.5, 1, -1)
    diag = np.array([np.searchsorted(ri[cp[j]:cp[j + 1]], j) + cp[j] for j in range(n)])
    lead[diag] += 8.0
    n_lanes = 333
    vals = np.stack([lead * rng.uniform(0.8, 1.2, nnz) for _ in range(n_lanes)])
    vals[5, diag[3]] = 0.0
    rhs = rng.normal(size=(n_lanes, n))
    ctx = lanes.DcLanes(fr)
    d_a = torch.tensor(vals.T.copy(), dtype=torch.float64, device="cuda")
    d_r = torch.tensor(rhs.T.copy(), dtype=torch.float64, device="cuda")
    out = []
    for call in (ctx.lu_lanes_mixed, ctx.lu_lanes_mixed_compiled):
        d_dx = torch.zeros((n, n_lanes), dtype=torch.float64, device="cuda")
        d_bad = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
        d_ref = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        call(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes, d_ref.data_ptr())
        torch.cuda.synchronize()
        out.append((d_dx.cpu().numpy().T, d_bad.cpu().numpy(), d_ref.cpu().numpy()))
    ctx.close()
    (dx_i, bad_i, ref_i), (dx_c, bad_c, ref_c) = out
    assert np.array_equal(bad_i, bad_c)
    good = bad_i == 0
    assert good.sum() > n_lanes // 2
    assert np.array_equal(ref_i[good], ref_c[good])
    assert np.all(np.abs(dx_c[good] - dx_i[good]) <= 1e-12 * np.abs(dx_i[good]).max(axis=1, keepdims=True))


@pytest.mark.parametrize("deck,seed", [("grid", 0), ("ring", 1)])
def test_lu_lanes_mixed_refines_to_fp64(deck, seed):
    """FP32 refactor and solves with FP64 refinement: dx within 1e-9 of the
    oracle's FP64 replay (the refinement drives the residual below 1e-12 of
    rhs), the same pivot-failure verdicts, at most a few corrections."""
    torch = _torch()
    fr = decks.grid_diodes(seed=seed + 1)[0] if deck == "grid" else decks.ring_oscillator(lanes=2)[0]
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(seed)
    lead = rng.uniform(0.5, 2.0, nnz) * np.where(rng.random(nnz) < 0.5, 1, -1)
    diag = np.array([np.searchsorted(ri[cp[j]:cp[j + 1]], j) + cp[j] for j in range(n)])
    lead[diag] += 8.0
    n_lanes = 333
    vals = np.stack([lead * rng.uniform(0.8, 1.2, nnz) for _ in range(n_lanes)])
    vals[0] = lead
    vals[5, diag[3]] = 0.0
    rhs = rng.normal(size=(n_lanes, n))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    ctx = lanes.DcLanes(fr)
    d_a = torch.tensor(vals.T.copy(), dtype=torch.float64, device="cuda")
    d_r = torch.tensor(rhs.T.copy(), dtype=torch.float64, device="cuda")
    d_dx = torch.zeros((n, n_lanes), dtype=torch.float64, device="cuda")
    d_bad = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
    d_ref = torch.zeros(n_lanes, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ctx.lu_lanes_mixed(lead, d_a.data_ptr(), d_r.data_ptr(), d_dx.data_ptr(), d_bad.data_ptr(), n_lanes,
                       d_ref.data_ptr())
    torch.cuda.synchronize()
    bad = d_bad.cpu().numpy()
    assert np.array_equal(bad, ref["bad"])
    good = bad == 0
    dx = d_dx.cpu().numpy().T
    assert _close(dx[good], ref["dx"][good]).all()
    refine = d_ref.cpu().numpy()[good]
    assert refine.max() <= 4 and refine.min() >= 1
    ctx.close()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_dc_lanes_match_oracle_warm(seed):
    fr, slots, values = decks.grid_diodes(seed=seed, points=256)
    opts_o = oracle.newton_opts()
    x0 = np.zeros(fr.n)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=x0, opts=opts_o)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    xg, itg, stg, stats = ctx.solve(x0=x0, opts=lanes.newton_opts())
    ctx.close()
    conv = stg == lanes.LANE_CONVERGED
    assert conv.all()
    bitwise = parity.assert_dc_parity(fr, slots, values, x0, opts_o, xg, itg, conv, xo, ito, cvo, f"seed {seed}")
    assert bitwise == 1.0, f"{bitwise:.3f} of the lanes bitwise the oracle's"
    assert stats["converged"] == 256


def test_dc_lanes_cold_start_match_oracle():
    fr, slots, values = decks.grid_diodes(seed=4, points=128)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    xg, itg, stg, stats = ctx.solve(x0=None)
    ctx.close()
    bitwise = parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(), xg, itg,
                                      stg == lanes.LANE_CONVERGED, xo, ito, cvo, "cold")
    assert bitwise == 1.0, f"{bitwise:.3f} of the lanes bitwise the oracle's"


def test_replicas_bitwise_identical():
    """tools/gpu_lane_parity.py's replica rule: equal lanes give equal bits."""
    fr, slots, _ = decks.grid_diodes(seed=5)
    values = np.full((64, 1), 3.3)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    xg, itg, stg, _ = ctx.solve(x0=np.zeros(fr.n))
    ctx.close()
    assert (xg.view(np.uint64) == xg[0].view(np.uint64)).all()
    assert (itg == itg[0]).all()


DC_FIXTURES = [n for n in gu.names("dc__") if "temp" not in n]

# Points in deep breakdown solved cold and independently: the reference's
# gates (converger.zig finalizeStep) judge a step assembled at the previous
# limited image, so a lane can pass them with its junction still limited
# (-8.8 V image, -18.5 V unknown). The oracle does the same; the reference
# reaches these points only warm, from its sequential sweep.
COLD_FALSE_CONVERGENCE = {"dc__device_diode_breakdown"}


@pytest.mark.parametrize("name", DC_FIXTURES)
def test_golden_fixtures_as_gpu_lanes(name):
    """Every sweep point of a reference fixture as an independent cold GPU
    lane: parity with the oracle's independent points at the deck's own
    options, and the reference's golden values at its tolerances when the
    lanes converge tightly (reltol 1e-6; a cold point at reltol 1e-3 is only
    that close to the answer)."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    inner = np.array(sweep_values(an[2], an[3], an[4]))
    slots = [fr.slot(an[1], "dc")]
    values = inner.reshape(-1, 1)
    if len(an) > 5:  # nested source sweep: one lane per (outer, inner) point
        outer = np.array(sweep_values(an[6], an[7], an[8]))
        slots.append(fr.slot(an[5], "dc"))
        values = np.stack([np.tile(inner, len(outer)), np.repeat(outer, len(inner))], axis=1)
    opts = deck.newton_opts()
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    x, it, st, _ = ctx.solve(x0=None, opts=lanes.newton_opts(**opts))
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None, opts=oracle.newton_opts(**opts))
    parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(**opts), x, it,
                            st == lanes.LANE_CONVERGED, xo, ito, cvo, name)
    if name in COLD_FALSE_CONVERGENCE:
        ctx.close()
        return
    tight = dict(opts, reltol=min(opts["reltol"], 1e-6))
    x, it, st, _ = ctx.solve(x0=None, opts=lanes.newton_opts(**tight))
    ctx.close()
    assert (st == lanes.LANE_CONVERGED).all()
    for col, worst, count in gu.score(g, fr, x):
        assert worst <= 1.0, f"{name} {col}: {worst:.3g}x the fixture tolerance"


def _fixture_points(name):
    """A reference DC fixture as independent points: (frozen, slots, values, opts)."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    values = np.array(sweep_values(an[2], an[3], an[4])).reshape(-1, 1)
    return fr, [fr.slot(an[1], "dc")], values, deck.newton_opts()


def test_device_entry_serves_pauses_on_caller_buffers():
    """esl_dc_solve_device with the caller's own status and iteration arrays,
    on a zener regulator swept into breakdown, whose lanes leave the lead
    pivot tape: the host factors the paused lanes from the caller's arrays
    (lane_solver.zig peels), the resumed lanes end as esl_dc_solve's (the
    context's own arrays) bit for bit, and both match the oracle."""
    torch = _torch()
    fr, slots, values, opts = _fixture_points("dc__bench_power_zener_reg")
    lo = lanes.newton_opts(**opts)
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, values)
    xh, ith, sth, st_h = ctx.solve(x0=None, opts=lo)
    N = len(values)
    d_x = torch.zeros((N, fr.n), dtype=torch.float64, device="cuda")
    d_it = torch.full((N,), 7, dtype=torch.int32, device="cuda")
    d_st = torch.full((N,), 9, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st_d = ctx.solve_device(d_x.data_ptr(), d_it.data_ptr(), d_st.data_ptr(), cold=True, opts=lo)
    torch.cuda.synchronize()
    xd, itd, std = d_x.cpu().numpy(), d_it.cpu().numpy().astype(np.uint32), d_st.cpu().numpy().astype(np.uint32)
    ctx.close()
    assert st_d["peeled"] > 0 and st_d["host_solves"] > 0, st_d
    assert st_d["peeled"] == st_h["peeled"] and st_d["host_solves"] == st_h["host_solves"]
    assert not (std == lanes.LANE_NEED_SOLVE).any()
    assert np.array_equal(std, sth) and np.array_equal(itd, ith)
    assert np.array_equal(xd.view(np.uint64), xh.view(np.uint64))
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None, opts=oracle.newton_opts(**opts))
    parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(**opts), xd, itd,
                            std == lanes.LANE_CONVERGED, xo, ito, cvo, "zener, caller buffers")

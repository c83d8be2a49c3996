"""Block lanes (a CTA per lane, block.cu) against the oracle on the B200.

- FP64: the same plain form as the warp lanes, so the same contract: every
  lane's converged flag and Newton iteration count exactly the oracle's, its
  solution bitwise the oracle's (the refactor and solves replay the pivot
  tape in the reference's order; the device models share the oracle's
  exp/log/pow). On the grid-with-diodes deck the block lanes also equal the
  warp lanes bit for bit.
- The circuits the warp lanes refuse (a working set beyond a warp's share of
  shared memory): the reference's 257-section resistor chain and 32 x 32
  grid fixtures, solved at their fixtures' tolerances; the analog block
  (about 500 unknowns, 120 BSIM3 devices) and all eight uneven-batch
  topologies (50 to 2,000 unknowns, the largest with its working set in
  global memory) on lane samples, against the oracle.
- Mixed precision (FP32 factors, FP64 refinement of every Newton step): each
  lane converges as the oracle's does, and its solution lies within 1e-9
  relative or 1e-12 absolute of the FP64 oracle's; iteration counts may
  differ (the refined step is not bitwise the FP64 step) and are reported.
- Lanes that leave the lead tape pause and take the host's factor on the
  block path too.
"""

import numpy as np
import pytest

import golden_util as gu
import parity
from espice_b200 import decks, lanes
from netlist import Deck
from oracle import oracle

pytestmark = pytest.mark.gpu


def _solve(fr, slots, values, x0=None, precision=lanes.PREC_FP64, path=lanes.PATH_BLOCK, opts=None):
    ctx = lanes.DcLanes(fr)
    ctx.set_mode(precision=precision, path=path)
    ctx.set_lanes(slots, values)
    x, it, st, stats = ctx.solve(x0=x0, opts=opts or lanes.newton_opts())
    info = ctx.block_info() if stats["path"] == lanes.PATH_BLOCK else None
    ctx.close()
    return x, it, st, stats, info


def test_block_fp64_equals_warp_and_oracle():
    fr, slots, values = decks.grid_diodes(seed=2, points=128)
    x0 = np.zeros(fr.n)
    xw, itw, stw, sw, _ = _solve(fr, slots, values, x0=x0, path=lanes.PATH_WARP)
    xb, itb, stb, sb, _ = _solve(fr, slots, values, x0=x0, path=lanes.PATH_BLOCK)
    assert sw["path"] == lanes.PATH_WARP and sb["path"] == lanes.PATH_BLOCK
    assert np.array_equal(stw, stb) and np.array_equal(itw, itb)
    assert np.array_equal(xw.view(np.uint64), xb.view(np.uint64))
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=x0)
    bitwise = parity.assert_dc_parity(fr, slots, values, x0, oracle.newton_opts(), xb, itb,
                                      stb == lanes.LANE_CONVERGED, xo, ito, cvo, "block")
    assert bitwise == 1.0


def test_block_fp64_bsim3_cold_bitwise():
    fr, slots, values = decks.bsim3_inverters(seed=1, lanes=96)
    xb, itb, stb, _, _ = _solve(fr, slots, values)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None)
    bitwise = parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(), xb, itb,
                                      stb == lanes.LANE_CONVERGED, xo, ito, cvo, "bsim3 block")
    assert bitwise == 1.0


@pytest.mark.parametrize("name", ["stress__scaling_resistor_grid_32x32", "convergence__resistor_chain_257"])
def test_fixtures_beyond_the_warp_lanes(name):
    """The fixtures the warp lanes refuse run on the block lanes (the
    automatic path), converge, and meet the fixture's tolerances."""
    g = gu.load(name)
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    opts = dict(deck.newton_opts(), reltol=1e-6)
    x, it, st, stats, info = _solve(fr, [], np.zeros((1, 1)), path=lanes.PATH_AUTO,
                                    opts=lanes.newton_opts(max_iter=100, **opts))
    assert stats["path"] == lanes.PATH_BLOCK and not info["warp_ok"]
    assert st[0] == lanes.LANE_CONVERGED, (int(st[0]), int(it[0]))
    xo, ito, cvo = oracle.dc_points(fr, [], np.zeros((1, 1)), warm=None, opts=oracle.newton_opts(max_iter=100, **opts))
    assert int(it[0]) == int(ito[0])
    assert np.array_equal(x.view(np.uint64), xo.view(np.uint64))
    for col, worst, count in gu.score(g, fr, x[:1]):
        assert worst <= 1.0, f"{name} {col}: {worst:.3g}x the fixture tolerance"


def _analog(points, seed=1):
    fr, expand = decks.analog_block()
    params, nominal = decks.analog_block_params(seed=seed, points=points)
    xn, _, cvn = oracle.dc_points(fr, expand.slots, expand(nominal), warm=None)
    assert cvn.all()
    return fr, expand.slots, expand(params), xn[0]


def test_analog_block_fp64_against_oracle():
    """48 points of the analog block from the nominal operating point."""
    fr, slots, values, x_nom = _analog(48)
    xb, itb, stb, stats, info = _solve(fr, slots, values, x0=x_nom, path=lanes.PATH_AUTO)
    assert stats["path"] == lanes.PATH_BLOCK
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=x_nom)
    bitwise = parity.assert_dc_parity(fr, slots, values, x_nom, oracle.newton_opts(), xb, itb,
                                      stb == lanes.LANE_CONVERGED, xo, ito, cvo, "analog block")
    assert bitwise == 1.0
    assert (stb == lanes.LANE_CONVERGED).all()


def test_analog_block_mixed_within_tolerance():
    fr, slots, values, x_nom = _analog(48, seed=2)
    xm, itm, stm, stats, info = _solve(fr, slots, values, x0=x_nom, precision=lanes.PREC_MIXED)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=x_nom)
    assert np.array_equal(stm == lanes.LANE_CONVERGED, cvo.astype(bool))
    ok = parity.close(xm, xo)
    assert ok.all(), float(np.max(np.abs(xm - xo) / (1e-12 + np.abs(xo))))
    assert stats["refinements"] > 0
    flips = int((itm != ito).sum())
    print(f"mixed: {flips} of {len(itm)} lanes took another iteration count; "
          f"{stats['refinements'] / len(itm):.2f} refinement corrections per lane")


@pytest.mark.parametrize("size", decks.MESH_GATES_SIZES)
def test_mesh_gates_topology_fp64_and_mixed(size):
    """Each uneven-batch topology on 12 supply values: FP64 bitwise the
    oracle's, mixed within the parity tolerance. The two largest keep their
    working set in global memory."""
    fr, slots = decks.mesh_gates(size)
    values = np.linspace(0.8, 1.8, 12).reshape(-1, 1)
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None)
    xb, itb, stb, stats, info = _solve(fr, slots, values)
    bitwise = parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(), xb, itb,
                                      stb == lanes.LANE_CONVERGED, xo, ito, cvo, f"mesh {size}")
    assert bitwise == 1.0
    if size >= 1500:
        assert not info["in_smem"][0]
    xm, itm, stm, _, _ = _solve(fr, slots, values, precision=lanes.PREC_MIXED)
    assert np.array_equal(stm == lanes.LANE_CONVERGED, cvo.astype(bool))
    conv = cvo.astype(bool)
    assert parity.close(xm[conv], xo[conv]).all(), float(np.max(np.abs(xm[conv] - xo[conv])))


def test_block_lanes_serve_pauses():
    """The zener regulator swept into breakdown on the block lanes: lanes
    leave the lead tape, pause, take the host's factor and resume; every
    lane matches the oracle exactly, as on the warp lanes."""
    g = gu.load("dc__bench_power_zener_reg")
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    an = deck.analysis
    from netlist import sweep_values
    values = np.array(sweep_values(an[2], an[3], an[4])).reshape(-1, 1)
    slots = [fr.slot(an[1], "dc")]
    opts = deck.newton_opts()
    xb, itb, stb, stats, _ = _solve(fr, slots, values, opts=lanes.newton_opts(**opts))
    assert stats["path"] == lanes.PATH_BLOCK and stats["peeled"] > 0, stats
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=None, opts=oracle.newton_opts(**opts))
    parity.assert_dc_parity(fr, slots, values, None, oracle.newton_opts(**opts), xb, itb,
                            stb == lanes.LANE_CONVERGED, xo, ito, cvo, "zener block")


def test_analog_block_mixed_adaptive_refinement():
    """Mixed precision with refine_skip: steps more than 1e3 tolerances from
    convergence go unrefined (inexact Newton), the rest are refined. Every
    point still converges as the oracle's does, within 1e-9 relative or
    1e-12 absolute of the FP64 oracle at the 1e-9 setting, with fewer
    refinement corrections than refining every step."""
    tight = dict(reltol=1e-9, vntol=1e-12, abstol=1e-15)
    fr, slots, values, x_nom = _analog(48, seed=4)
    refs = {}
    for skip in (0.0, 1e3):
        ctx = lanes.DcLanes(fr)
        ctx.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=skip)
        ctx.set_lanes(slots, values)
        xm, itm, stm, stats = ctx.solve(x0=x_nom, opts=lanes.newton_opts(**tight))
        ctx.close()
        refs[skip] = stats["refinements"]
        xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=x_nom, opts=oracle.newton_opts(**tight))
        assert np.array_equal(stm == lanes.LANE_CONVERGED, cvo.astype(bool))
        ok = parity.close(xm, xo)
        assert ok.all(), float(np.max(np.abs(xm - xo) / (1e-12 + np.abs(xo))))
        print(f"refine_skip {skip:g}: {stats['refinements']} corrections, iterations {itm.mean():.2f} "
              f"(oracle {ito.mean():.2f})")
    assert refs[1e3] < refs[0.0]


def test_mesh_gates_20k_unknowns_slab_lanes():
    """A 20,001-unknown mesh with 1,666 BSIM3 gates (the large transient
    configuration's size) as 16 DC lanes with the working set in the per-CTA
    global slab: every lane converges, two lanes bitwise the oracle's with
    the same iteration counts."""
    fr, slots = decks.mesh_gates(20000)
    values = np.linspace(0.8, 1.8, 16).reshape(-1, 1)
    xb, itb, stb, stats, info = _solve(fr, slots, values)
    assert fr.n == 20001 and not info["in_smem"][0]
    assert (stb == lanes.LANE_CONVERGED).all()
    xo, ito, cvo = oracle.dc_points(fr, slots, values[:2], warm=None)
    assert cvo.all() and np.array_equal(itb[:2], ito)
    assert np.array_equal(xb[:2].view(np.uint64), xo.view(np.uint64))
    print(f"20k lanes: {stats['kernel_ms']:.1f} ms for 16 lanes, {itb.mean():.2f} iterations, "
          f"{info['a_rows']} rows in program A over {info['a_levels']} levels")


def test_live_parameter_lanes_equal_expanded_lanes():
    """esl_set_lanes_cols: the analog block's points given as their 16 live
    parameters with the slot-to-column map solve bitwise as the same points
    given as their 248 expanded slot values, with the same iteration counts,
    and both equal the oracle's."""
    fr, expand = decks.analog_block()
    params, nominal = decks.analog_block_params(seed=6, points=24)
    out = []
    for cols in (None, expand.cols):
        ctx = lanes.DcLanes(fr)
        ctx.set_mode(path=lanes.PATH_BLOCK)
        ctx.set_lanes(expand.slots, expand(params) if cols is None else expand.lane_params(params), cols=cols)
        out.append(ctx.solve(x0=None))
        ctx.close()
    (xa, ita, sta, _), (xb, itb, stb, _) = out
    assert np.array_equal(xa.view(np.uint64), xb.view(np.uint64))
    assert np.array_equal(ita, itb) and np.array_equal(sta, stb)
    xo, ito, cvo = oracle.dc_points(fr, expand.slots, expand(params), warm=None)
    assert np.array_equal(stb == lanes.LANE_CONVERGED, cvo.astype(bool))
    assert np.array_equal(itb, ito)
    assert np.array_equal(xb.view(np.uint64), xo.view(np.uint64))

"""The points API (include/espice_points.h) on the B200 against the oracle.

A points problem mirrors the reference's espice_append_points /
espice_copy_point_measures / espice_release_points (include/espice.h:286-360):
points appended in batches run as lanes when their results are first copied.

- Transient points with .meas cards (ring oscillator): every point's card
  values within 1e-9 of the oracle's streamed measures (the tolerance of the
  measure tests), reasons MEASURE_UNRESOLVED exactly where a requested card
  has no value; early_stop changes no value.
- Operating-point points (grid with diodes), cold and warm from the
  template's nominal operating point: unknowns bitwise the oracle's.
- A point's results do not depend on the batch it ran in or its lane width.
- The reference's error codes: unknown names, ids outside the appended
  points, released points, a short options struct, tangents, abort_after.
"""

import math

import numpy as np
import pytest

from espice_b200 import decks, lanes, points
from oracle import oracle

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-9, 1e-15
NAMES = ["period", "delay", "tfall", "last", "find", "win_rise", "vmax", "vmin", "vavg", "vpp"]


def _cards(fr, mod):
    s0, s5 = fr.unknown("v(s0)"), fr.unknown("v(s5)")
    return [
        mod.Measure(mod.MEAS_TRIG_TARG, 0, mod.meas_clause(s0, val=0.9, rise=2),
                    mod.meas_clause(s0, val=0.9, rise=3)),
        mod.Measure(mod.MEAS_TRIG_TARG, 0, mod.meas_clause(s0, val=0.9, cross=3),
                    mod.meas_clause(s5, val=0.9, cross=3)),
        mod.Measure(mod.MEAS_WHEN, 0, mod.meas_clause(s0, val=0.9, fall=1, td=0.2e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_WHEN, 0, mod.meas_clause(s5, val=0.5, cross=mod.MEAS_LAST), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_FIND_AT, 0, mod.meas_clause(s5, at=0.37e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_WHEN, 0, mod.meas_clause(s0, val=0.9, rise=1, from_=0.5e-9, to=1.5e-9),
                    mod.meas_clause(0)),
        mod.Measure(mod.MEAS_MAX, 0, mod.meas_clause(s0, from_=1e-9, to=2e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_MIN, 0, mod.meas_clause(s5, from_=0.5e-9, to=2.5e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_AVG, 0, mod.meas_clause(s0, from_=1e-9), mod.meas_clause(0)),
        mod.Measure(mod.MEAS_PP, 0, mod.meas_clause(s5, from_=1e-9), mod.meas_clause(0)),
    ]


def _same(a, b):
    both_nan = np.isnan(a) & np.isnan(b)
    return both_nan | (np.abs(a - b) <= ATOL + RTOL * np.maximum(np.abs(a), np.abs(b)))


def _tran_problem(fr, slots, lane_width=0):
    results = [(n.upper() if k % 2 else n, points.RESULT_MEASURE, k) for k, n in enumerate(NAMES)]
    return points.Points(fr, slots, points.TRAN, results, measures=_cards(fr, lanes),
                         tran=lanes.tran_opts(3e-9, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=200_000),
                         lane_width=lane_width)


@pytest.mark.parametrize("early", [False, True])
def test_tran_points_match_oracle(early):
    """20 ring-oscillator points appended as 7 + 13, run as lane batches of
    8; names copied in another order and case."""
    fr, slots, values = decks.ring_oscillator(lanes=20)
    P = _tran_problem(fr, slots, lane_width=8)
    assert P.lane_width() == 8
    opts = points.options(early_stop=early)
    a = P.append(values[:7], opts)
    b = P.append(values[7:], opts)
    assert (a, b) == (0, 7)
    order = [3, 0, 9, 1, 4, 2, 5, 8, 6, 7]
    got, reasons = P.copy_measures(0, 20, [NAMES[k].title() for k in order])
    P.close()
    vo, so, _ = oracle.tran_meas(fr, slots, values, oracle.tran_opts(3e-9, decks.RING_T_STEP, decks.RING_T_MAX,
                                                                      max_steps=200_000),
                                 _cards(fr, oracle), early_stop=early)
    want = vo[:, order]
    same = _same(got, want)
    assert same.all(), (got[~same], want[~same])
    unresolved = np.isnan(want).any(axis=1)
    assert np.array_equal(reasons == points.REASON_MEASURE_UNRESOLVED, unresolved)
    assert np.all(reasons[~unresolved] == points.REASON_OK)
    assert np.isfinite(got[:, order.index(0)]).any()


def test_points_do_not_depend_on_batching():
    """The same 6 points in one batch of lane width 6 and one at a time:
    bitwise the same card values."""
    fr, slots, values = decks.ring_oscillator(lanes=6)
    P = _tran_problem(fr, slots, lane_width=6)
    P.append(values)
    whole, r1 = P.copy_measures(0, 6, NAMES)
    P.close()
    Q = _tran_problem(fr, slots, lane_width=1)
    Q.append(values)
    single, r2 = Q.copy_measures(0, 6, NAMES)
    Q.close()
    assert np.array_equal(r1, r2)
    assert np.array_equal(np.nan_to_num(whole, nan=7.0).view(np.uint64),
                          np.nan_to_num(single, nan=7.0).view(np.uint64))


@pytest.mark.parametrize("warm", [False, True])
def test_op_points_match_oracle(warm):
    """48 grid-with-diodes points (three appends), five unknowns each: cold
    from the zero start, or warm from the template's nominal operating
    point, bitwise the oracle's."""
    fr, slots, values = decks.grid_diodes(seed=3, points=48)
    pick = [1, 5, 17, 30, fr.n - 1]
    results = [(f"x{k}", points.RESULT_UNKNOWN, k) for k in pick]
    P = points.Points(fr, slots, points.OP, results, newton=lanes.newton_opts())
    opts = points.options(warm_start=warm)
    P.append(values[:10], opts)
    P.append(values[10:40], opts)
    P.append(values[40:], opts)
    got, reasons = P.copy_measures(0, 48, [f"X{k}" for k in pick])
    P.close()
    x0 = None
    if warm:
        xn, _, cvn = oracle.dc_points(fr, [], np.zeros((1, 1)), warm=None)
        assert cvn.all()
        x0 = xn[0]
    xo, ito, cvo = oracle.dc_points(fr, slots, values, warm=x0)
    assert np.array_equal(reasons == points.REASON_OK, cvo.astype(bool))
    conv = cvo.astype(bool)
    assert np.array_equal(got[conv].view(np.uint64), xo[conv][:, pick].view(np.uint64))
    assert np.isnan(got[~conv]).all()


def test_points_errors():
    fr, slots, values = decks.grid_diodes(seed=3, points=4)
    P = points.Points(fr, slots, points.OP, [("x1", points.RESULT_UNKNOWN, 1)])
    with pytest.raises(points.PointsError) as e:
        P.append(values, points.options(struct_size=32))
    assert e.value.code == points.PTS_ABI_MISMATCH
    for bad in (points.options(tangent_step=1e-3), points.options(abort_after=1e-9),
                points.options(abort_after=-1.0), points.options(abort_after=math.inf)):
        with pytest.raises(points.PointsError) as e:
            P.append(values, bad)
        assert e.value.code == points.PTS_INVALID_ARGUMENT
    # the 40-byte layout (no tangent_step) is accepted
    first = P.append(values, points.options(struct_size=40))
    assert first == 0
    with pytest.raises(points.PointsError) as e:
        P.copy_measures(0, 4, ["nope"])
    assert e.value.code == points.PTS_INVALID_ARGUMENT
    with pytest.raises(points.PointsError) as e:
        P.copy_measures(2, 3, ["x1"])
    assert e.value.code == points.PTS_INVALID_QUERY
    v, r = P.copy_measures(0, 4, ["X1"])
    assert (r == points.REASON_OK).all() and np.isfinite(v).all()
    P.release(0, 2)
    with pytest.raises(points.PointsError) as e:
        P.copy_measures(0, 4, ["x1"])
    assert e.value.code == points.PTS_RESULT_UNAVAILABLE
    v2, _ = P.copy_measures(2, 2, ["x1"])
    assert np.array_equal(v2, v[2:])
    P.close()

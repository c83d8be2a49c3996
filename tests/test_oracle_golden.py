"""The oracle against the reference's own golden fixtures (ngspice-44.2 and
analytic oracles, scored at the reference's per-column tolerances)."""

import pytest

import golden_util as gu
from oracle import oracle


def _dc(fr, slot, values, opts):
    return oracle.dc_sweep(fr, slot, values, oracle.newton_opts(**opts))


def _op(fr, opts):
    return oracle.op(fr, oracle.newton_opts(max_iter=100, **opts))


DC_OP = [n for n in gu.names() if not n.startswith("tran")]


@pytest.mark.parametrize("name", DC_OP)
def test_oracle_matches_golden(name):
    g = gu.load(name)
    fr, rows, conv = gu.solve_deck(g, _dc, _op)
    assert conv.all(), f"{name}: {int((~conv.astype(bool)).sum())} points did not converge"
    for col, worst, count in gu.score(g, fr, rows):
        assert worst <= 1.0, f"{name} {col}: error {worst:.3g}x the allowed tolerance"


TRAN = [n for n in gu.names("tran__") if gu.load(n)["plots"]]
MEAS = [n for n in gu.names("tran__") if gu.load(n).get("checks")]


@pytest.mark.parametrize("name", TRAN)
def test_oracle_transient_matches_golden(name):
    """The transient restatement against the reference's ngspice-44.2
    waveform: the oracle's accepted points, linearly interpolated at the
    fixture's sample times, within each column's tolerance."""
    g = gu.load(name)
    fr, t, v, cols, st = gu.solve_tran(g)
    assert st["status"] == 0, st
    for col, worst in gu.score_tran(g, t, v, cols):
        assert worst <= 1.0, f"{name} {col}: error {worst:.3g}x the allowed tolerance"


@pytest.mark.parametrize("name", MEAS)
def test_oracle_measures_match_golden(name):
    """The streamed .meas cards of a transient fixture against the values
    ngspice printed, at the fixture's tolerance."""
    g = gu.load(name)
    values, st = gu.solve_meas(g)
    assert st[0] == 0, st
    for nm, worst in gu.score_meas(g, values):
        assert worst <= 1.0, f"{name} {nm}: error {worst:.3g}x the allowed tolerance"


def test_mos1_tox_is_dc_only():
    """MOS1 with TOX: DC solves (TOX enters only KP's default: u0 * Cox'),
    the transient is refused, as the library refuses it (the bias-dependent
    Meyer halves and their $prev averaging are not built)."""
    import numpy as np
    from espice_b200.circuit import Circuit
    c = Circuit()
    c.V("vdd", "d", "0", dc=1.8)
    c.V("vg", "g", "0", dc=1.2)
    c.M("m1", "d", "g", "0", "0", type=1.0, vto=0.5, tox=20e-9, u0=400.0, w=2e-6, l=1e-6)
    fr = c.freeze()
    x, it, cv = oracle.dc_points(fr, [], np.zeros((1, 1)), warm=None)
    assert cv[0]
    # the drain current at KP = u0 * 3.9 eps0 / tox * 1e-4 (saturation, lambda
    # 0), beside the drain junction's gmin leak (1e-12 S at 1.8 V)
    kp = 400.0 * 3.9 * 8.854214871e-12 / 20e-9 * 1e-4
    want = 0.5 * kp * 2.0 * (1.2 - 0.5) ** 2
    assert abs(-x[0, fr.unknown("i(vdd)")] - want) <= 1e-6 * want
    with pytest.raises(ValueError):
        oracle.tran(fr, [], np.zeros((1, 1)), oracle.tran_opts(1e-9, 1e-11))

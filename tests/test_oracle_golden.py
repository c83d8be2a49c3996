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

"""Test helper: runs a golden fixture deck through the oracle (or a library
entry point with the same signature) and scores it as the reference does:
|got - expected| <= atol + rtol * |expected| per column
(tests/test_correctness.zig:625-627), on the selected rows."""

import glob
import json
import os

import numpy as np

from netlist import Deck, sweep_values

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        return json.load(fh)


def names(prefix=""):
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.json"))):
        n = os.path.basename(p)[:-5]
        if n.startswith(prefix):
            out.append(n)
    return out


def solve_deck(g, dc_sweep, op):
    """Returns (frozen, rows [n_rows][n]) for the deck's analysis."""
    deck = Deck(g["deck"])
    ckt = deck.circuit()
    an = deck.analysis
    if an[0] == "op":
        fr = ckt.freeze()
        x, it, rc = op(fr, deck.newton_opts())
        return fr, x[None, :], np.array([rc == 0])
    assert an[0] == "dc"
    inner = sweep_values(an[2], an[3], an[4])
    outer = [None]
    if len(an) > 5:
        outer = sweep_values(an[6], an[7], an[8])
    rows, conv = [], []
    fr = None
    for ov in outer:
        if ov is not None and an[5] == "temp":
            ckt.set_temp(ov)
        fr = ckt.freeze()
        if ov is not None and an[5] != "temp":
            # nested source sweep: the outer source's bias, in place
            ob = fr.slot(an[5], "dc")
            fr.batches[ob.batch][2][ob.inst, ob.param] = ov
        slot = fr.slot(an[1], "dc")
        x, it, cv = dc_sweep(fr, slot, np.array(inner), deck.newton_opts())
        rows.append(x)
        conv.append(cv)
    return fr, np.concatenate(rows), np.concatenate(conv)


def score(g, fr, rows):
    """List of (column, worst ratio err/allowed, n checked)."""
    out = []
    for plot in g["plots"]:
        idx = plot.get("row_indices") or list(range(plot["row_count"]))
        for col, spec in plot["columns"].items():
            k = fr.unknown(col)
            got = rows[idx, k]
            exp = np.array(spec["values"], dtype=float)
            allowed = spec["atol"] + spec["rtol"] * np.abs(exp)
            err = np.abs(got - exp)
            out.append((col, float(np.max(err / allowed)), len(exp)))
    return out


def solve_tran(g, max_pts=1_000_000):
    """Runs a .tran fixture through the oracle: (frozen, t, v [pts][cols],
    columns, stats dict)."""
    from oracle import oracle
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    _, tstep, tstop, tstart, tmax = deck.analysis
    assert tstart == 0.0, "a TSTART after 0 is not supported"
    assert deck.options.get("method", "trap") == "trap", "the trapezoidal integrator only"
    cols = list(g["plots"][0]["columns"])
    probes = [fr.unknown(c) for c in cols]
    o = oracle.tran_opts(tstop, tstep, tmax, **deck.newton_opts())
    t, v, npts, stats, _ = oracle.tran(fr, [], np.zeros((1, 1)), o, probes, max_pts=max_pts)
    n = int(npts[0])
    return fr, t[0, :n], v[0, :n], cols, dict(zip(oracle.TS_FIELDS, stats[0].tolist()))


def score_tran(g, t, v, cols):
    """(column, worst err/allowed) with the waveform interpolated at the
    fixture's sample times."""
    plot = g["plots"][0]
    at = np.array(plot["axis"]["values"])
    out = []
    for k, col in enumerate(cols):
        spec = plot["columns"][col]
        exp = np.array(spec["values"], dtype=float)
        got = np.interp(at, t, v[:, k])
        allowed = spec["atol"] + spec["rtol"] * np.abs(exp)
        out.append((col, float(np.max(np.abs(got - exp) / allowed))))
    return out


def measure_cards(deck, fr, mod):
    """The deck's .meas cards as `mod`'s Measure structs (mod: the library's
    lanes module or the oracle)."""
    kinds = {"when": mod.MEAS_WHEN, "trig_targ": mod.MEAS_TRIG_TARG, "find_at": mod.MEAS_FIND_AT}
    out = []
    for m in deck.measures:
        cl = [mod.meas_clause(fr.unknown(c["vec"]), val=c["val"], rise=c["rise"], fall=c["fall"],
                              cross=c["cross"], td=c["td"], from_=c["from"], to=c["to"], at=c["at"])
              for c in m["clauses"]]
        while len(cl) < 2:
            cl.append(mod.meas_clause(0))
        out.append(mod.Measure(kinds[m["kind"]], 0, cl[0], cl[1]))
    return out


def tran_options(deck):
    """The .tran card's options for tran_opts: (tstop, tstep, tmax, kwargs)."""
    _, tstep, tstop, tstart, tmax = deck.analysis
    assert tstart == 0.0, "a TSTART after 0 is not supported"
    kw = dict(deck.newton_opts())
    for k in ("chgtol", "trtol"):
        if k in deck.options:
            kw[k] = deck.options[k]
    return tstop, tstep, tmax, kw


def solve_meas(g):
    """The fixture's .meas cards through the oracle's transient: {name: value}."""
    from oracle import oracle
    deck = Deck(g["deck"])
    fr = deck.circuit().freeze()
    tstop, tstep, tmax, kw = tran_options(deck)
    o = oracle.tran_opts(tstop, tstep, tmax, max_steps=2_000_000, **kw)
    v, st, _ = oracle.tran_meas(fr, [], np.zeros((1, 1)), o, measure_cards(deck, fr, oracle))
    return {m["name"]: float(v[0, k]) for k, m in enumerate(deck.measures)}, st[0]


def score_meas(g, values):
    """(name, err / allowed) for every measure check of the fixture."""
    out = []
    for c in g.get("checks", []):
        got = values[c["name"].lower()]
        allowed = c["atol"] + c["rtol"] * abs(c["value"])
        out.append((c["name"], abs(got - c["value"]) / allowed))
    return out

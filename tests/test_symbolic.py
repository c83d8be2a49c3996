"""Host-only checks of the library's symbolic stage against the oracle:
the frozen pattern, the column order, the lead pivot tape, and the
level-scheduled warp programs (emulated on the CPU) bitwise equal to the
reference's column replay of the refactor and solves."""

import numpy as np
import pytest

import golden_util as gu
import program_emu as emu
from espice_b200 import decks, lanes
from netlist import Deck
from oracle import oracle


def _random_mna(n, seed, density=0.08):
    """sparse_lu.zig TestSystem-style random pattern: full diagonal, circuit
    sparsity, 15% zero diagonals on columns with another entry."""
    rng = np.random.default_rng(seed)
    cols = []
    for j in range(n):
        rows = {j} | {i for i in range(n) if i != j and rng.random() < density}
        cols.append(sorted(rows))
    cp = np.zeros(n + 1, np.uint32)
    ri, vals = [], []
    for j, rows in enumerate(cols):
        s = 0.0
        entries = []
        for i in rows:
            v = rng.uniform(-1, 1) if i != j else 0.0
            s += abs(v)
            entries.append((i, v))
        zero_diag = len(rows) > 1 and rng.random() < 0.15
        for i, v in entries:
            ri.append(i)
            vals.append((0.0 if zero_diag else s + 1.0) if i == j else v)
        cp[j + 1] = len(ri)
    return cp, np.array(ri, np.uint32), np.array(vals)


def _lead_matrix(frozen):
    """A lane-0-like Jacobian on the pattern: the oracle's first assembly."""
    cp, ri = oracle.pattern(frozen)
    return cp, ri


DECKS = ["dc__bench_ensemble_sweep_lanes", "convergence__diode_stack_8",
         "stress__scaling_resistor_grid_32x32", "convergence__bench_diode_bridge",
         "dc__bench_mosfet_cmos_inverter", "dc__device_mos1_output", "tran__device_mos1_large_signal"]


@pytest.mark.parametrize("name", DECKS)
def test_pattern_matches_oracle(name):
    fr = Deck(gu.load(name)["deck"]).circuit().freeze()
    cp_o, ri_o = oracle.pattern(fr)
    cp_l, ri_l = lanes.pattern(fr)
    assert np.array_equal(cp_o, cp_l) and np.array_equal(ri_o, ri_l)


def test_grid_diode_pattern_and_order():
    fr, slots, values = decks.grid_diodes()
    cp, ri = oracle.pattern(fr)
    assert np.array_equal(cp, lanes.pattern(fr)[0])
    q_o = oracle.order(fr.n, cp, ri)
    rng = np.random.default_rng(3)
    vals = rng.uniform(0.5, 2.0, len(ri))
    tape = lanes.compile_tape(fr.n, cp, ri, vals)
    rc, ot = oracle.factor_tape(fr.n, cp, ri, vals)
    assert rc == 0
    assert np.array_equal(q_o, ot["q"])
    assert np.array_equal(tape["q"], ot["q"])
    assert np.array_equal(tape["pinv"], ot["pinv"])


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("n", [5, 17, 40, 64])
def test_programs_bitwise_oracle_replay(n, seed):
    cp, ri, lead = _random_mna(n, seed)
    rc, ot = oracle.factor_tape(n, cp, ri, lead)
    if rc != 0:
        pytest.skip("singular draw")
    tape = lanes.compile_tape(n, cp, ri, lead)
    assert tape["info"]["has_void"] == 0
    assert np.array_equal(tape["q"], ot["q"]) and np.array_equal(tape["pinv"], ot["pinv"])
    assert tape["info"]["nl"] == len(ot["li"]) and tape["info"]["nu"] == len(ot["ui"])
    rng = np.random.default_rng(seed + 100)
    lanes_n = 4
    vals = np.stack([lead * rng.uniform(0.9, 1.1, len(lead)) for _ in range(lanes_n)])
    vals[0] = lead
    rhs = rng.normal(size=(lanes_n, n))
    ref = oracle.lane_refactor_solve(n, cp, ri, lead, vals, rhs)
    nu = tape["info"]["nu"]
    for l in range(lanes_n):
        tv, dx, bad = emu.refactor_solve(tape, vals[l], rhs[l], n)
        assert bad == bool(ref["bad"][l])
        if bad:
            continue
        assert np.array_equal(tv[:nu].view(np.uint64), ref["ux"][l].view(np.uint64))
        assert np.array_equal(tv[nu:nu + n].view(np.uint64), ref["udiag"][l].view(np.uint64))
        assert np.array_equal(tv[nu + n:nu + n + len(ot["li"])].view(np.uint64),
                              ref["lx"][l].view(np.uint64))
        assert np.array_equal(dx.view(np.uint64), ref["dx"][l].view(np.uint64))


def test_program_levels_shorter_than_sequence():
    fr, _, _ = decks.grid_diodes()
    cp, ri = oracle.pattern(fr)
    rng = np.random.default_rng(5)
    tape = lanes.compile_tape(fr.n, cp, ri, rng.uniform(0.5, 2.0, len(ri)))
    info = tape["info"]
    assert info["a_levels"] < info["a_nops"] and info["a_rows"] * 32 >= info["a_nops"]
    assert info["b_levels"] < info["b_nops"] and info["b_rows"] * 32 >= info["b_nops"]

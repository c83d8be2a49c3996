"""Regenerates tests/golden/*.json from the reference's own fixture corpus.

Each golden file holds one reference deck (its .sp text) and the oracle
values the reference checks it against (its .expected.json: ngspice-44.2 or
analytic columns, with the per-column tolerances the reference scores at,
tests/test_correctness.zig:397-398). Run in a container that has the
reference checked out; the outputs are committed so tests never read it.

    python tests/golden/make_golden.py /path/to/reference
"""

import json
import os
import sys

FIXTURES = [
    # DC sweeps: R, V, I, diode
    "dc/bench_ensemble_sweep_lanes",
    "dc/bench_dc_sweep_vin_sweep",
    "dc/device_diode_iv_sweep",
    "dc/device_diode_breakdown",
    "dc/diode_forward",
    "dc/diode_reverse",
    "dc/diode_reverse_continuation",
    "dc/bench_power_zener_reg",
    "convergence/bench_mos_latch_ladder",
    "dc/device_diode_temp",
    # operating points
    "convergence/diode_stack_8",
    "convergence/bench_diode_bridge",
    "convergence/diode_knee",
    "convergence/diode_emission_two",
    "convergence/diode_forward",
    "convergence/diode_high_current",
    "convergence/diode_large_is",
    "convergence/diode_reverse",
    "convergence/diode_small_is",
    "convergence/diode_stack_2",
    "convergence/diode_stack_32",
    "convergence/diode_weak_current",
    "convergence/diode_zero",
    "convergence/resistor_chain_8",
    "convergence/resistor_chain_31",
    "convergence/resistor_chain_64",
    "convergence/resistor_chain_257",
    "op/bench_medium_resistor_mesh",
    "stress/scaling_resistor_grid_32x32",
    # MOS1
    "dc/device_mos1_transfer",
    "dc/device_mos1_output",
    "dc/bench_mosfet_cmos_inverter",
    "tran/device_mos1_large_signal",
    "dc/device_mos1_body_effect",
    "dc/device_mos1_pmos",
    "dc/device_mos1_subthreshold",
    "dc/bench_sweep_cmos_inv_sizing",
    "dc/device_mos1_temp",
    # BSIM3v3 DC core (LEVEL 49)
    "dc/device_bsim3_transfer",
    "dc/device_bsim3_output",
    "dc/device_bsim3_body_effect",
    "dc/device_bsim3_pmos",
    "dc/device_bsim3_temp",
    "op/device_bsim3",
    # transients: RC networks and MOS1 under PULSE sources
    "tran/bench_tran_rc_pulse",
    "tran/bench_medium_rc_ladder_50",
    "tran/bench_digital_rc_filter_chain",
    "tran/bench_digital_buffer_rc",
    "tran/bench_mosfet_nmos_cs",
    "tran/rc_pulse_history_trap",
    "tran/finite_rise_positive",
    # transients under SIN, EXP and PWL sources (V and I)
    "tran/sine",
    "tran/sine_offset_phase",
    "tran/rc_sinusoidal_startup",
    "tran/bench_tran_exp_source",
    "tran/source_exp_defaults_ngspice",
    "tran/pwl_triangle",
    "tran/pwl_nonzero_start",
    "tran/pwl_isource_breakpoints",
    # transient measures (FIND .. AT=) against ngspice's printed values
    "tran/zero_abstol_vntol",
    "tran/zero_vntol_chgtol",
]


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    for f in FIXTURES:
        base = os.path.join(ref, "tests", "fixtures", f)
        with open(base + ".sp") as fh:
            deck = fh.read()
        with open(base + ".expected.json") as fh:
            exp = json.load(fh)
        out = {
            "source": "tests/fixtures/" + f + ".sp",
            "deck": deck,
            "analysis": exp["analysis"],
            "oracle": exp["oracle"]["kind"],
            "plots": exp["expect"].get("plots", []),
            "checks": [c for c in exp["expect"].get("checks", []) if c.get("kind") == "measure"],
        }
        name = f.replace("/", "__") + ".json"
        with open(os.path.join(here, name), "w") as fh:
            json.dump(out, fh, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout (the directory holding tests/fixtures)>")
    main(sys.argv[1])

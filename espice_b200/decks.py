"""Seeded synthetic decks of the sweep-lane workloads (the reference has no
public suite for this path; these stand in with the stated shapes, sizes and
value distributions, and fixed seeds).

grid_diodes: an 8x8 resistor grid (R log-uniform in [100, 10k] ohm), 16
diodes (IS = 1e-14 A, N = 1, RS = 10 ohm) from seeded grid nodes to ground
and one voltage source at the corner node, swept 0..5 V in 256 points. About
82 unknowns with the diodes' internal nodes and the source's branch row.

ring_oscillator: a 31-stage CMOS ring of MOS1 inverters (NMOS KP = 120u,
VTO = 0.45, LAMBDA = 0.05; PMOS KP = 40u, VTO = -0.45, LAMBDA = 0.05;
W/L = 1u/0.18u), 10 fF load per stage, VDD = 1.8 V brought up by a 50 ps
supply ramp from 0 V at t = 0 (the operating point is all-zero and the ring
leaves its metastable point on the devices' mismatch, not on rounding). Each
lane draws every device's VTO from N(nominal, 30 mV). 34 unknowns. The
transient is trapezoidal to 20 ns with a 1 ps maximum step.

bsim3_inverters: a chain of CMOS inverters of BSIM3v3 (LEVEL 49) devices,
L = 0.18 um, VDD = 1.8 V, each output loaded by 50 kohm to ground. The NMOS
cards cycle through three variants so every branch of the DC core runs:
the ngspice-fixture card (given VTH0, K1, K2), a card with the k1/k2 ladder
and the vfb/vth0 defaults derived, RSH series resistance (internal drain and
source nodes), impact ionisation (ALPHA0) and poly depletion (NGATE) under
MOBMOD 2, and a MOBMOD 3 card. Each lane draws the input voltage from
U(0, VDD) and every device's DELVTO from N(0, 20 mV).
"""

from __future__ import annotations

import numpy as np

from .circuit import B3, M, Circuit


def grid_diodes(seed: int = 1, rows: int = 8, cols: int = 8, n_diodes: int = 16,
                points: int = 256, v_stop: float = 5.0):
    """Returns (frozen circuit, [source dc slot], sweep values [points][1])."""
    rng = np.random.default_rng(seed)
    c = Circuit()
    name = lambda r, k: f"n{r}_{k}"  # noqa: E731
    c.V("vin", name(0, 0), "0", dc=0.0)
    for r in range(rows):
        for k in range(cols):
            if k + 1 < cols:
                c.R(f"rh{r}_{k}", name(r, k), name(r, k + 1), float(np.exp(rng.uniform(np.log(100), np.log(1e4)))))
            if r + 1 < rows:
                c.R(f"rv{r}_{k}", name(r, k), name(r + 1, k), float(np.exp(rng.uniform(np.log(100), np.log(1e4)))))
    nodes = rng.choice(rows * cols, size=n_diodes, replace=False)
    for i, nd in enumerate(sorted(int(v) for v in nodes)):
        c.D(f"d{i}", name(nd // cols, nd % cols), "0", is_=1e-14, n=1.0, rs=10.0)
    fr = c.freeze()
    slot = fr.slot("vin", "dc")
    values = np.linspace(0.0, v_stop, points).reshape(-1, 1)
    return fr, [slot], values


def grid_diodes_16(seed: int = 1, points: int = 65536):
    """The grid-with-diodes deck with 16 swept parameters per point (the
    learned warm start's workload): the corner source uniform in [0, 5] V and
    15 grid resistors each scaled by exp(U(-0.7, 0.7)) from seed. Returns
    (frozen, 16 slots, values [points][16], nominal values [16])."""
    fr, slots, _ = grid_diodes(seed=1)
    rng = np.random.default_rng(seed + 1000)
    rs = [s for s in fr.slots_of(0, "r")][:15]
    slots = list(slots) + rs
    nominal = np.array([fr.param(s) for s in slots])
    nominal[0] = 2.5
    values = np.empty((points, len(slots)))
    values[:, 0] = rng.uniform(0.0, 5.0, points)
    values[:, 1:] = nominal[1:] * np.exp(rng.uniform(-0.7, 0.7, size=(points, len(slots) - 1)))
    return fr, slots, values, nominal


RING_T_STOP = 20e-9
RING_T_STEP = 1e-12
RING_T_MAX = 1e-12


def ring_oscillator(seed: int = 1, stages: int = 31, lanes: int = 1024, sigma: float = 0.03,
                    vdd: float = 1.8, c_load: float = 10e-15, ramp: float = 50e-12):
    """Returns (frozen circuit, per-device vto slots, values [lanes][2 * stages])."""
    rng = np.random.default_rng(seed)
    c = Circuit()
    c.V("vdd", "vdd", "0", dc=0.0, pulse=[0.0, vdd, 0.0, ramp, ramp, 1.0, 2.0])
    for k in range(stages):
        inp, out = f"s{(k - 1) % stages}", f"s{k}"
        c.M(f"mn{k}", out, inp, "0", "0", type=1.0, vto=0.45, kp=120e-6, **{"lambda": 0.05}, w=1e-6, l=0.18e-6)
        c.M(f"mp{k}", out, inp, "vdd", "vdd", type=-1.0, vto=-0.45, kp=40e-6, **{"lambda": 0.05}, w=1e-6,
            l=0.18e-6)
        c.C(f"cl{k}", out, "0", c_load)
    fr = c.freeze()
    slots = fr.slots_of(M, "vto")
    nominal = np.array([fr.batches[s.batch][2][s.inst, s.param] for s in slots])
    values = nominal + rng.normal(0.0, sigma, size=(lanes, len(slots)))
    return fr, slots, values


# BSIM3v3 cards (LEVEL 49): the NMOS of the reference's ngspice fixtures and
# two variants, and the fixtures' PMOS.
B3_NMOS = [
    dict(type=1.0, tox=4.1e-9, vth0=0.35, k1=0.53, k2=-0.06, k3=80.0, vsat=1.5e5, ua=-1.4e-9, ub=2.3e-18,
         uc=-4.6e-11, rdsw=200.0, u0=280.0, pclm=1.3, pdiblc1=0.39, pdiblc2=0.0086),
    dict(type=1.0, mobmod=2.0, tox=4.1e-9, nch=2.3e17, vsat=1.4e5, u0=300.0, rdsw=150.0, rsh=20.0, nrd=1.0,
         nrs=1.0, alpha0=1e-6, beta0=25.0, ngate=5e19),
    dict(type=1.0, mobmod=3.0, tox=4.1e-9, vth0=0.4, k1=0.5, k2=-0.05, u0=260.0, ua=1.0e-9, ub=1.0e-18,
         vsat=1.2e5, rdsw=250.0),
]
B3_PMOS = dict(type=-1.0, tox=4.1e-9, vth0=-0.4, k1=0.55, k2=-0.05, k3=80.0, vsat=1.2e5, ua=-1.4e-9,
               ub=2.3e-18, uc=-4.6e-11, rdsw=400.0, u0=100.0, pclm=1.3, pdiblc1=0.39, pdiblc2=0.0086)


def bsim3_inverters(seed: int = 1, stages: int = 6, lanes: int = 256, sigma: float = 0.02,
                    vdd: float = 1.8, r_load: float = 50e3, c_load: float = 0.0, pulse=None):
    """Returns (frozen circuit, [input dc slot] + per-device delvto slots,
    values [lanes][1 + 2 * stages]). c_load > 0 adds a capacitor to ground
    on every output and `pulse` (a PULSE list) drives the input, for a
    transient (the BSIM3 DC core has no charges of its own)."""
    rng = np.random.default_rng(seed)
    c = Circuit()
    c.V("vdd", "vdd", "0", dc=vdd)
    c.V("vin", "s_in", "0", dc=0.0, pulse=pulse)
    prev = "s_in"
    for k in range(stages):
        out = f"s{k}"
        c.B3(f"mn{k}", out, prev, "0", "0", w=2e-6, l=0.18e-6, **B3_NMOS[k % len(B3_NMOS)])
        c.B3(f"mp{k}", out, prev, "vdd", "vdd", w=4e-6, l=0.18e-6, **B3_PMOS)
        c.R(f"rl{k}", out, "0", r_load)
        if c_load > 0.0:
            c.C(f"cl{k}", out, "0", c_load)
        prev = out
    fr = c.freeze()
    from .circuit import V
    slots = [fr.slots_of(V, "dc")[1]] + fr.slots_of(B3, "delvto")
    values = np.empty((lanes, len(slots)))
    values[:, 0] = rng.uniform(0.0, vdd, lanes)
    values[:, 1:] = rng.normal(0.0, sigma, size=(lanes, len(slots) - 1))
    return fr, slots, values

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

analog_block (the learned warm start's workload): a seeded BSIM3 analog
block of 120 MOSFETs on a 20 x 21 RC mesh (R log-uniform in [100, 10k] ohm
between neighbours, C log-uniform in [1, 100] fF to ground, the mesh's edge
nodes tied to VREF through 1 kohm): twenty 5-transistor OTAs (an NMOS
differential pair with a PMOS current-mirror load and an NMOS tail mirror),
each a unity-gain follower whose input is a seeded mesh node and whose output
drives another seeded mesh node through 2 kohm; a bias network of six current
sources, each into a diode-connected NMOS (the tails' mirror gates) and
mirrored into a diode-connected PMOS; an NMOS source follower on the last
OTA. About 500 unknowns. 16 parameters per point, uniform from seed: VDD in
[1.6, 2.0] V, VREF in [0.8, 1.0] V, the six bias currents log-uniform in
[1, 100] uA, the temperature in [-40, 125] C (every device), and seven DELVTO
shifts in [-50, 50] mV (device k takes shift k mod 7).

mesh_gates (the uneven batch): eight seeded topologies of about 50 to 2,000
unknowns, each a planar RC mesh (R log-uniform in [10, 10k] ohm, C in
[1, 100] fF to ground) with BSIM3 (LEVEL 49 card defaults, L = 0.18 um,
W log-uniform in [0.2, 2] um) inverters and NAND2 gates, one per twelve
unknowns, each at a seeded mesh node (its output) with its inputs on mesh
nodes within two rows and columns of it; two mesh nodes tied to ground and to
the supply through 1 kohm. Each lane is one supply value in [0.8, 1.8] V.
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


ANALOG_PARAMS = ["vdd", "vref"] + [f"ibias{k}" for k in range(6)] + ["temp_c"] + [f"dvto{k}" for k in range(7)]


def analog_block(seed: int = 1, rows: int = 20, cols: int = 21, n_ota: int = 20):
    """The analog block at its nominal parameters. Returns (frozen circuit,
    expand) where expand(params [points][16]) gives the lane values for the
    slots expand.slots (the two sources' dc, the six bias currents, then
    every device's temperature in K and its DELVTO)."""
    rng = np.random.default_rng(seed)
    c = Circuit()
    c.V("vdd", "vdd", "0", dc=1.8)
    c.V("vref", "vref", "0", dc=0.9)
    mesh = lambda r, k: f"m{r}_{k}"  # noqa: E731
    for r in range(rows):
        for k in range(cols):
            if k + 1 < cols:
                c.R(f"rh{r}_{k}", mesh(r, k), mesh(r, k + 1), float(np.exp(rng.uniform(np.log(100), np.log(1e4)))))
            if r + 1 < rows:
                c.R(f"rv{r}_{k}", mesh(r, k), mesh(r + 1, k), float(np.exp(rng.uniform(np.log(100), np.log(1e4)))))
            c.C(f"cm{r}_{k}", mesh(r, k), "0", float(np.exp(rng.uniform(np.log(1e-15), np.log(1e-13)))))
            if r in (0, rows - 1) or k in (0, cols - 1):
                c.R(f"re{r}_{k}", mesh(r, k), "vref", 1e3)
    nm = dict(B3_NMOS[0])
    pm = dict(B3_PMOS)

    def nmos(name, d, g, s_, w):
        c.B3(name, d, g, s_, "0", w=w, l=0.18e-6, **nm)

    def pmos(name, d, g, s_, w):
        c.B3(name, d, g, s_, "vdd", w=w, l=0.18e-6, **pm)

    # bias network: I_k into a diode NMOS (nb_k), mirrored into a diode PMOS (pb_k)
    for k in range(6):
        c.I(f"ib{k}", "vdd", f"nb{k}", dc=10e-6)
        nmos(f"mbn{k}", f"nb{k}", f"nb{k}", "0", 2e-6)
        nmos(f"mbm{k}", f"pb{k}", f"nb{k}", "0", 2e-6)
        pmos(f"mbp{k}", f"pb{k}", f"pb{k}", "vdd", 4e-6)
    interior = [(r, k) for r in range(1, rows - 1) for k in range(1, cols - 1)]
    picks = rng.choice(len(interior), size=2 * n_ota, replace=False)
    for o in range(n_ota):
        a = mesh(*interior[picks[2 * o]])
        b = mesh(*interior[picks[2 * o + 1]])
        t, mm, out = f"t{o}", f"l{o}", f"o{o}"
        nmos(f"m1_{o}", mm, a, t, 4e-6)      # + input
        nmos(f"m2_{o}", out, out, t, 4e-6)   # - input tied to the output
        pmos(f"m3_{o}", mm, mm, "vdd", 8e-6)
        pmos(f"m4_{o}", out, mm, "vdd", 8e-6)
        nmos(f"m5_{o}", t, f"nb{o % 6}", "0", 4e-6)
        c.R(f"ro{o}", out, b, 2e3)
    # source follower on the last OTA's output
    nmos("msf", "vdd", f"o{n_ota - 1}", "sf", 4e-6)
    nmos("msk", "sf", "nb0", "0", 2e-6)
    fr = c.freeze()
    from .circuit import I as I_, V as V_
    vsl = fr.slots_of(V_, "dc")
    isl = fr.slots_of(I_, "dc")
    tsl = fr.slots_of(B3, "temp")
    dsl = fr.slots_of(B3, "delvto")
    n_dev = len(tsl)
    group = np.arange(n_dev) % 7

    def expand(params):
        params = np.atleast_2d(np.asarray(params, np.float64))
        out = np.empty((params.shape[0], 2 + 6 + 2 * n_dev))
        out[:, 0:2] = params[:, 0:2]
        out[:, 2:8] = params[:, 2:8]
        out[:, 8:8 + n_dev] = params[:, 8:9] + 273.15
        out[:, 8 + n_dev:] = params[:, 9 + group]
        return out

    def lane_params(params):
        """The points' 16 parameters as the lanes' live parameter values
        (esl_set_lanes_cols): the temperature in kelvin, the rest as given;
        slot s takes column expand.cols[s]."""
        out = np.array(params, np.float64, ndmin=2, copy=True)
        out[:, 8] += 273.15
        return out

    expand.slots = list(vsl) + list(isl) + list(tsl) + list(dsl)
    expand.cols = np.concatenate([np.arange(8), np.full(n_dev, 8), 9 + np.asarray(group)]).astype(np.uint32)
    expand.lane_params = lane_params
    expand.n_devices = n_dev
    return fr, expand


def analog_block_params(seed: int = 1, points: int = 65536):
    """The 16 parameters of `points` analog-block points, uniform from seed:
    [points][16] in ANALOG_PARAMS order, and the nominal point [16]."""
    rng = np.random.default_rng(seed + 4000)
    p = np.empty((points, 16))
    p[:, 0] = rng.uniform(1.6, 2.0, points)
    p[:, 1] = rng.uniform(0.8, 1.0, points)
    p[:, 2:8] = np.exp(rng.uniform(np.log(1e-6), np.log(100e-6), size=(points, 6)))
    p[:, 8] = rng.uniform(-40.0, 125.0, points)
    p[:, 9:16] = rng.uniform(-0.05, 0.05, size=(points, 7))
    nominal = np.array([1.8, 0.9] + [10e-6] * 6 + [27.0] + [0.0] * 7)
    return p, nominal


MESH_GATES_SIZES = [50, 100, 200, 400, 700, 1000, 1500, 2000]


def mesh_gates(size: int, seed: int = 1):
    """One uneven-batch topology of about `size` unknowns. Returns (frozen
    circuit, [supply dc slot])."""
    rng = np.random.default_rng(seed * 7919 + size)
    n_gates = max(2, size // 12)
    # mesh nodes: the size less the NAND2 internal nodes and the supply's node and branch
    n_mesh = max(9, size - n_gates // 2 - 2)
    cols = int(np.ceil(np.sqrt(n_mesh)))
    c = Circuit()
    c.V("vdd", "vdd", "0", dc=1.8)
    mesh = lambda i: f"m{i}"  # noqa: E731
    for i in range(n_mesh):
        r, k = divmod(i, cols)
        if k + 1 < cols and i + 1 < n_mesh:
            c.R(f"rh{i}", mesh(i), mesh(i + 1), float(np.exp(rng.uniform(np.log(10), np.log(1e4)))))
        if i + cols < n_mesh:
            c.R(f"rv{i}", mesh(i), mesh(i + cols), float(np.exp(rng.uniform(np.log(10), np.log(1e4)))))
        c.C(f"cm{i}", mesh(i), "0", float(np.exp(rng.uniform(np.log(1e-15), np.log(1e-13)))))
    c.R("rtie0", mesh(0), "0", 1e3)
    c.R("rtie1", mesh(n_mesh - 1), "vdd", 1e3)
    card_n = dict(type=1.0)
    card_p = dict(type=-1.0)
    def near(i):
        # a mesh node within two rows and columns of node i (a gate's pins
        # are near each other on the layout), not i itself
        r, k = divmod(i, cols)
        while True:
            rr = int(np.clip(r + rng.integers(-2, 3), 0, (n_mesh - 1) // cols))
            kk = int(np.clip(k + rng.integers(-2, 3), 0, cols - 1))
            j = rr * cols + kk
            if j != i and j < n_mesh:
                return j

    for g in range(n_gates):
        w = float(np.exp(rng.uniform(np.log(0.2e-6), np.log(2e-6))))
        centre = int(rng.integers(n_mesh))
        a1 = near(centre)
        a2 = near(centre)
        while a2 == a1:
            a2 = near(centre)
        ins = [mesh(a1), mesh(a2), mesh(centre)]
        out = ins[2]
        if g % 2 == 0:  # inverter
            c.B3(f"mn{g}", out, ins[0], "0", "0", w=w, l=0.18e-6, **card_n)
            c.B3(f"mp{g}", out, ins[0], "vdd", "vdd", w=2 * w, l=0.18e-6, **card_p)
        else:  # NAND2
            mid = f"x{g}"
            c.B3(f"mna{g}", out, ins[0], mid, "0", w=w, l=0.18e-6, **card_n)
            c.B3(f"mnb{g}", mid, ins[1], "0", "0", w=w, l=0.18e-6, **card_n)
            c.B3(f"mpa{g}", out, ins[0], "vdd", "vdd", w=2 * w, l=0.18e-6, **card_p)
            c.B3(f"mpb{g}", out, ins[1], "vdd", "vdd", w=2 * w, l=0.18e-6, **card_p)
    fr = c.freeze()
    return fr, [fr.slot("vdd", "dc")]


C5_T_STOP = 5e-9


def digital_block(size: int = 20000, seed: int = 5, n_cells: int = 500, n_inputs: int = 16,
                  t_stop: float = C5_T_STOP):
    """The large transient configuration's circuit: a seeded digital block of
    n_cells BSIM3 NAND2 cells (4 MOSFETs each: 2,000 at the default) on a
    planar RC parasitic mesh (R log-uniform 10 ohm - 10 kohm, C 1 - 100 fF),
    about `size` unknowns, driven by n_inputs seeded piecewise-linear pulse
    trains (0 to 1.8 V, 50 ps edges, through 50 ohm into mesh nodes) over
    t_stop. Returns (frozen circuit, the MOSFETs' DELVTO slots)."""
    rng = np.random.default_rng(seed * 104729 + size)
    n_mesh = max(16, size - n_cells - 2 * n_inputs - 2)
    cols = int(np.ceil(np.sqrt(n_mesh)))
    c = Circuit()
    c.V("vdd", "vdd", "0", dc=1.8)
    mesh = lambda i: f"m{i}"  # noqa: E731
    for i in range(n_mesh):
        r, k = divmod(i, cols)
        if k + 1 < cols and i + 1 < n_mesh:
            c.R(f"rh{i}", mesh(i), mesh(i + 1), float(np.exp(rng.uniform(np.log(10), np.log(1e4)))))
        if i + cols < n_mesh:
            c.R(f"rv{i}", mesh(i), mesh(i + cols), float(np.exp(rng.uniform(np.log(10), np.log(1e4)))))
        c.C(f"cm{i}", mesh(i), "0", float(np.exp(rng.uniform(np.log(1e-15), np.log(1e-13)))))
    c.R("rtie0", mesh(0), "0", 1e3)
    c.R("rtie1", mesh(n_mesh - 1), "vdd", 1e3)
    edge = 50e-12
    for k in range(n_inputs):
        # a pulse train: a seeded first edge, then widths and gaps of 0.2-1 ns
        pts, t, level = [(0.0, 0.0)], float(rng.uniform(0.02e-9, 0.5e-9)), 0.0
        while t + edge < t_stop and len(pts) < 60:
            pts.append((t, level))
            level = 1.8 - level
            pts.append((t + edge, level))
            t += edge + float(rng.uniform(0.2e-9, 1.0e-9))
        c.V(f"vin{k}", f"in{k}", "0", pwl=([p[0] for p in pts], [p[1] for p in pts]))
        c.R(f"rin{k}", f"in{k}", mesh(int(rng.integers(n_mesh))), 50.0)

    def near(i):
        r, k = divmod(i, cols)
        while True:
            rr = int(np.clip(r + rng.integers(-2, 3), 0, (n_mesh - 1) // cols))
            kk = int(np.clip(k + rng.integers(-2, 3), 0, cols - 1))
            j = rr * cols + kk
            if j != i and j < n_mesh:
                return j

    card_n = dict(type=1.0)
    card_p = dict(type=-1.0)
    names = []
    for g in range(n_cells):
        w = float(np.exp(rng.uniform(np.log(0.2e-6), np.log(2e-6))))
        out = int(rng.integers(n_mesh))
        a = near(out)
        b = near(out)
        while b == a:
            b = near(out)
        mid = f"x{g}"
        c.B3(f"mna{g}", mesh(out), mesh(a), mid, "0", w=w, l=0.18e-6, **card_n)
        c.B3(f"mnb{g}", mid, mesh(b), "0", "0", w=w, l=0.18e-6, **card_n)
        c.B3(f"mpa{g}", mesh(out), mesh(a), "vdd", "vdd", w=2 * w, l=0.18e-6, **card_p)
        c.B3(f"mpb{g}", mesh(out), mesh(b), "vdd", "vdd", w=2 * w, l=0.18e-6, **card_p)
        names += [f"mna{g}", f"mnb{g}", f"mpa{g}", f"mpb{g}"]
    fr = c.freeze()
    return fr, [fr.slot(nm, "delvto") for nm in names]


def digital_block_vto(n_devices: int, lanes: int, seed: int = 7, sigma: float = 0.02):
    """Per-device threshold shifts of the large transient configuration's
    lanes: DELVTO ~ N(0, sigma) per MOSFET and lane, [lanes][n_devices]."""
    return np.random.default_rng(seed).normal(0.0, sigma, size=(lanes, n_devices))

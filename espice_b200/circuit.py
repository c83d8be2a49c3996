"""Circuit description for the sweep-lane library: unknown numbering and the
per-type instance tables the C ABI (``include/espice_lanes.h``) takes.

This is the host half of the reference's frozen circuit
(``src/device/Circuit.zig:77-167``): node 0 is ground and is row/column 0 of
the matrix, held by a unit pin; every other unknown is an external node, a
device-internal node (a diode's ``ai`` behind RS, a MOSFET's ``di``/``si``
behind RD/RS) or a voltage source's branch current. External nodes are
numbered in order of first use, then internal unknowns in batch order.

Device tables mirror the Verilog-A parameter lists the reference compiles
(``models/{resistor,capacitor,vsource,isource,diode,mos1,bsim3}.va``). Values are
the card values; bias-independent temperature maps run in the library.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

R, C, V, I, D, M, B3 = 0, 1, 2, 3, 4, 5, 6
NODES_PER = {R: 2, C: 2, V: 3, I: 2, D: 3, M: 6, B3: 6}

# Diode parameter slots (models/diode.va:35-103).
D_PARAMS = ["is", "n", "rs", "bv", "ibv", "cjo", "vj", "m", "fc", "tt", "area",
            "gmin", "xti", "eg", "tnom", "temp"]
D_DEFAULTS = dict(is_=1e-14, n=1.0, rs=0.0, bv=0.0, ibv=1e-3, cjo=0.0, vj=1.0, m=0.5,
                  fc=0.5, tt=0.0, area=1.0, gmin=1e-12, xti=3.0, eg=1.11, tnom=27.0,
                  temp=300.15)

# MOS1 parameter slots (models/mos1.va:20-85); type +1 NMOS, -1 PMOS.
M_PARAMS = ["type", "vto", "kp", "gamma", "phi", "lambda", "rd", "rs", "cbd", "cbs",
            "is", "pb", "cgso", "cgdo", "cgbo", "cj", "mj", "cjsw", "mjsw", "tox",
            "ld", "u0", "fc", "w", "l", "ad", "as", "pd", "ps", "delvto", "m", "gmin",
            "tnom", "temp"]
# KP NaN: not given (its default is u0 * Cox' with TOX given, else 2e-5).
M_DEFAULTS = {"type": 1.0, "vto": 0.0, "kp": float("nan"), "gamma": 0.0, "phi": 0.6, "lambda": 0.0,
              "rd": 0.0, "rs": 0.0, "cbd": 0.0, "cbs": 0.0, "is": 1e-14, "pb": 0.8,
              "cgso": 0.0, "cgdo": 0.0, "cgbo": 0.0, "cj": 0.0, "mj": 0.5, "cjsw": 0.0,
              "mjsw": 0.5, "tox": 0.0, "ld": 0.0, "u0": 600.0, "fc": 0.5, "w": 1e-4,
              "l": 1e-4, "ad": 0.0, "as": 0.0, "pd": 0.0, "ps": 0.0, "delvto": 0.0,
              "m": 1.0, "gmin": 1e-12, "tnom": 27.0, "temp": 300.15}

# BSIM3v3 DC-core parameter slots (models/bsim3.va:26-138: the model card,
# then the instance, then gmin and the device temperature in K). NaN marks a
# parameter left off the card whose default the model derives
# ($param_given): TOXM, NCH, GAMMA1, GAMMA2, VBX, K1, K2, VTH0, VFB, DSUB,
# UC, UC1, U0.
B3_PARAMS = ["type", "mobmod", "tnom", "tox", "toxm", "xj", "nch", "nsub", "ngate", "gamma1",
             "gamma2", "xt", "vbx", "vbm", "k1", "k2", "k3", "k3b", "w0", "nlx", "vth0", "vfb",
             "dvt0", "dvt1", "dvt2", "dvt0w", "dvt1w", "dvt2w", "drout", "dsub", "nfactor",
             "cdsc", "cdscb", "cdscd", "cit", "vsat", "at", "a0", "ags", "a1", "a2", "keta",
             "ua", "ua1", "ub", "ub1", "uc", "uc1", "u0", "ute", "voff", "delta", "rdsw",
             "prwg", "prwb", "prt", "wr", "eta0", "etab", "pclm", "pdiblc1", "pdiblc2",
             "pdiblcb", "pscbe1", "pscbe2", "pvag", "dwg", "dwb", "b0", "b1", "alpha0",
             "alpha1", "beta0", "kt1", "kt1l", "kt2", "lint", "ll", "lln", "lw", "lwn", "lwl",
             "wint", "wl", "wln", "ww", "wwn", "wwl", "xl", "xw", "js", "jsw", "nj", "xti",
             "ijth", "rsh", "l", "w", "ad", "as", "pd", "ps", "nrd", "nrs", "m", "delvto",
             "mulu0", "gmin", "temp"]
_NAN = float("nan")
B3_DEFAULTS = {
    "type": 1.0, "mobmod": 1.0, "tnom": 27.0, "tox": 150.0e-10, "toxm": _NAN, "xj": 0.15e-6,
    "nch": _NAN, "nsub": 6.0e16, "ngate": 0.0, "gamma1": _NAN, "gamma2": _NAN, "xt": 1.55e-7,
    "vbx": _NAN, "vbm": -3.0, "k1": _NAN, "k2": _NAN, "k3": 80.0, "k3b": 0.0, "w0": 2.5e-6,
    "nlx": 1.74e-7, "vth0": _NAN, "vfb": _NAN, "dvt0": 2.2, "dvt1": 0.53, "dvt2": -0.032,
    "dvt0w": 0.0, "dvt1w": 5.3e6, "dvt2w": -0.032, "drout": 0.56, "dsub": _NAN,
    "nfactor": 1.0, "cdsc": 2.4e-4, "cdscb": 0.0, "cdscd": 0.0, "cit": 0.0, "vsat": 8.0e4,
    "at": 3.3e4, "a0": 1.0, "ags": 0.0, "a1": 0.0, "a2": 1.0, "keta": -0.047, "ua": 2.25e-9,
    "ua1": 4.31e-9, "ub": 5.87e-19, "ub1": -7.61e-18, "uc": _NAN, "uc1": _NAN, "u0": _NAN,
    "ute": -1.5, "voff": -0.08, "delta": 0.01, "rdsw": 0.0, "prwg": 0.0, "prwb": 0.0,
    "prt": 0.0, "wr": 1.0, "eta0": 0.08, "etab": -0.07, "pclm": 1.3, "pdiblc1": 0.39,
    "pdiblc2": 0.0086, "pdiblcb": 0.0, "pscbe1": 4.24e8, "pscbe2": 1.0e-5, "pvag": 0.0,
    "dwg": 0.0, "dwb": 0.0, "b0": 0.0, "b1": 0.0, "alpha0": 0.0, "alpha1": 0.0, "beta0": 30.0,
    "kt1": -0.11, "kt1l": 0.0, "kt2": 0.022, "lint": 0.0, "ll": 0.0, "lln": 1.0, "lw": 0.0,
    "lwn": 1.0, "lwl": 0.0, "wint": 0.0, "wl": 0.0, "wln": 1.0, "ww": 0.0, "wwn": 1.0,
    "wwl": 0.0, "xl": 0.0, "xw": 0.0, "js": 1.0e-4, "jsw": 0.0, "nj": 1.0, "xti": 3.0,
    "ijth": 0.1, "rsh": 0.0, "l": 5.0e-6, "w": 5.0e-6, "ad": 0.0, "as": 0.0, "pd": 0.0,
    "ps": 0.0, "nrd": 1.0, "nrs": 1.0, "m": 1.0, "delvto": 0.0, "mulu0": 1.0, "gmin": 1e-12,
    "temp": 300.15}
# ngspice card spellings that name the same parameter
B3_ALIASES = {"npeak": "nch", "uo": "u0"}

# V and I sources (models/vsource.va, isource.va): dc, wave (0 DC, 1 PULSE,
# 2 SIN, 3 EXP, 4 PWL), the wave's eight parameters in slots 2..9 (named for
# PULSE: v1 v2 td tr tf pw per phase; SIN: vo va freq td theta phase; EXP: v1
# v2 td1 tau1 td2 tau2; PWL: len repeat td), then the PWL table: 64 times and
# 64 values.
PWL_MAX = 64
SRC_PARAMS = (["dc", "wave", "v1", "v2", "td", "tr", "tf", "pw", "per", "phase"]
              + [f"pwl_t{k}" for k in range(PWL_MAX)] + [f"pwl_v{k}" for k in range(PWL_MAX)])
V_PARAMS = SRC_PARAMS
WAVE = {"dc": 0, "pulse": 1, "sin": 2, "exp": 3, "pwl": 4}
PARAMS_PER = {R: 1, C: 1, V: len(SRC_PARAMS), I: len(SRC_PARAMS), D: len(D_PARAMS), M: len(M_PARAMS),
              B3: len(B3_PARAMS)}
PARAM_NAMES = {R: ["r"], C: ["c"], V: SRC_PARAMS, I: SRC_PARAMS, D: D_PARAMS, M: M_PARAMS,
               B3: B3_PARAMS}


def source_params(dc=0.0, pulse=None, sin=None, exp=None, pwl=None):
    """The 138 source parameters: dc and at most one wave. pulse: [v1 v2 td
    tr tf pw per phase] (missing ones take the model's -1 / 0 sentinels);
    sin: [vo va freq td theta phase]; exp: [v1 v2 td1 tau1 td2 tau2]; pwl:
    (times, values[, repeat, td]) with at most 64 points (repeat < 0: none)."""
    prm = [float(dc), 0.0] + [0.0] * 8 + [0.0] * (2 * PWL_MAX)
    if pulse is not None:
        prm[1] = 1.0
        vals = list(pulse) + [None] * (8 - len(pulse))
        defaults = [0.0, 0.0, 0.0, -1.0, -1.0, -1.0, -1.0, 0.0]
        for k in range(8):
            prm[2 + k] = float(vals[k]) if vals[k] is not None else defaults[k]
    elif sin is not None:
        prm[1] = 2.0
        vals = list(sin) + [0.0] * (6 - len(sin))
        prm[2:8] = [float(v) for v in vals[:6]]
    elif exp is not None:
        prm[1] = 3.0
        defaults = [0.0, 0.0, 0.0, 1.0e-9, 0.0, 1.0e-9]
        vals = list(exp) + [None] * (6 - len(exp))
        prm[2:8] = [float(v) if v is not None else d for v, d in zip(vals[:6], defaults)]
    elif pwl is not None:
        times, values = list(pwl[0]), list(pwl[1])
        repeat = float(pwl[2]) if len(pwl) > 2 else -1.0
        td = float(pwl[3]) if len(pwl) > 3 else 0.0
        if len(times) != len(values) or not 0 < len(times) <= PWL_MAX:
            raise ValueError(f"a PWL source takes 1 to {PWL_MAX} points")
        prm[1] = 4.0
        prm[2:5] = [float(len(times)), repeat, td]
        prm[10:10 + len(times)] = [float(v) for v in times]
        prm[10 + PWL_MAX:10 + PWL_MAX + len(values)] = [float(v) for v in values]
    return prm
TYPE_ORDER = [R, C, V, I, D, M, B3]
TYPE_LETTER = {R: "R", C: "C", V: "V", I: "I", D: "D", M: "M", B3: "M"}


@dataclass
class _Dev:
    name: str
    type: int
    ext: list          # external node names
    params: list
    internal: list = field(default_factory=list)  # "a"/"ai" markers resolved at freeze


class Circuit:
    """A netlist under construction; ``freeze`` numbers the unknowns."""

    def __init__(self, temp_c: float = 27.0):
        self.node_ids = {"0": 0, "gnd": 0}
        self.devs: list[_Dev] = []
        self.temp_k = temp_c + 273.15
        self._frozen = None

    def node(self, name) -> int:
        name = str(name).lower()
        if name not in self.node_ids:
            self.node_ids[name] = len([k for k in self.node_ids if k != "gnd"])
        return self.node_ids[name]

    def _add(self, name, typ, ext, params):
        for e in ext:
            self.node(e)
        self.devs.append(_Dev(name.lower(), typ, [str(e).lower() for e in ext], list(params)))
        self._frozen = None

    def R(self, name, p, n, r):
        self._add(name, R, [p, n], [float(r)])

    def C(self, name, p, n, c):
        self._add(name, C, [p, n], [float(c)])

    def V(self, name, p, n, dc=0.0, pulse=None, sin=None, exp=None, pwl=None):
        """A voltage source: dc and at most one wave (source_params)."""
        self._add(name, V, [p, n], source_params(dc, pulse, sin, exp, pwl))

    def I(self, name, p, n, dc=0.0, pulse=None, sin=None, exp=None, pwl=None):
        """A current source from p to n through the source (source_params)."""
        self._add(name, I, [p, n], source_params(dc, pulse, sin, exp, pwl))

    def D(self, name, a, c, area=1.0, **model):
        kw = dict(D_DEFAULTS)
        kw["temp"] = self.temp_k
        for k, v in model.items():
            k = k.lower()
            k = {"is": "is_", "js": "is_", "cj0": "cjo", "cj": "cjo", "mj": "m"}.get(k, k)
            if k not in kw:
                raise ValueError(f"diode parameter {k!r} is not supported")
            kw[k] = float(v)
        kw["area"] = float(area)
        prm = [kw["is_"] if p == "is" else kw[p] for p in D_PARAMS]
        self._add(name, D, [a, c], prm)

    def M(self, name, d, g, s, b, **params):
        kw = dict(M_DEFAULTS)
        kw["temp"] = self.temp_k
        given_tox = False
        for k, v in params.items():
            k = k.lower()
            k = {"uo": "u0", "lambda_": "lambda"}.get(k, k)
            if k not in kw:
                raise ValueError(f"mos1 parameter {k!r} is not supported")
            kw[k] = float(v)
            given_tox |= k == "tox"
        prm = [kw[p] for p in M_PARAMS]
        self._add(name, M, [d, g, s, b], prm)

    def B3(self, name, d, g, s, b, **params):
        """A BSIM3v3 MOSFET (LEVEL 8/49 card, DC core)."""
        kw = dict(B3_DEFAULTS)
        kw["temp"] = self.temp_k
        for k, v in params.items():
            k = B3_ALIASES.get(k.lower(), k.lower())
            if k not in kw:
                raise ValueError(f"bsim3 parameter {k!r} is not supported")
            kw[k] = float(v)
        self._add(name, B3, [d, g, s, b], [kw[p] for p in B3_PARAMS])

    def set_temp(self, temp_c):
        """Circuit temperature for every device without its own TEMP."""
        self.temp_k = temp_c + 273.15
        for d in self.devs:
            if d.type == D:
                d.params[D_PARAMS.index("temp")] = self.temp_k
            elif d.type == M:
                d.params[M_PARAMS.index("temp")] = self.temp_k
            elif d.type == B3:
                d.params[B3_PARAMS.index("temp")] = self.temp_k
        self._frozen = None

    # ------------------------------------------------------------------
    def freeze(self) -> "Frozen":
        if self._frozen is not None:
            return self._frozen
        n_ext = len([k for k in self.node_ids if k != "gnd"])
        nxt = n_ext
        names = {v: k for k, v in self.node_ids.items() if k != "gnd"}
        batches = {}
        where = {}
        current = []
        for t in TYPE_ORDER:
            devs = [d for d in self.devs if d.type == t]
            if not devs:
                continue
            nodes = np.zeros((len(devs), NODES_PER[t]), dtype=np.uint32)
            prm = np.zeros((len(devs), PARAMS_PER[t]), dtype=np.float64)
            for i, d in enumerate(devs):
                ext = [self.node_ids[e] for e in d.ext]
                if t == V:
                    ext.append(nxt)
                    names[nxt] = f"i({d.name})"
                    current.append(nxt)
                    nxt += 1
                elif t == D:
                    if d.params[D_PARAMS.index("rs")] > 0:
                        ext.append(nxt)
                        names[nxt] = f"{d.name}#ai"
                        nxt += 1
                    else:
                        ext.append(ext[0])
                elif t == M:
                    rd = d.params[M_PARAMS.index("rd")]
                    rs = d.params[M_PARAMS.index("rs")]
                    if rd > 0:
                        ext.append(nxt)
                        names[nxt] = f"{d.name}#di"
                        nxt += 1
                    else:
                        ext.append(ext[0])
                    if rs > 0:
                        ext.append(nxt)
                        names[nxt] = f"{d.name}#si"
                        nxt += 1
                    else:
                        ext.append(ext[2])
                elif t == B3:
                    # RSH times the squares NRD / NRS, else the node collapses
                    rsh = d.params[B3_PARAMS.index("rsh")]
                    for k, (sq, ref) in enumerate((("nrd", 0), ("nrs", 2))):
                        if rsh > 0 and d.params[B3_PARAMS.index(sq)] > 0:
                            ext.append(nxt)
                            names[nxt] = f"{d.name}#{'di' if k == 0 else 'si'}"
                            nxt += 1
                        else:
                            ext.append(ext[ref])
                nodes[i] = ext
                prm[i] = d.params
                where[d.name] = (len(batches), i)
            batches[t] = (nodes, prm)
        n = nxt
        cur = np.zeros(n, dtype=np.uint8)
        cur[current] = 1
        self._frozen = Frozen(n, [(t, *batches[t]) for t in batches], cur, names, where,
                              dict(self.node_ids))
        return self._frozen


class _Batch(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("nodes", ctypes.POINTER(ctypes.c_uint32)),
                ("params", ctypes.POINTER(ctypes.c_double))]


class _Circuit(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("n_batches", ctypes.c_uint32),
                ("batches", ctypes.POINTER(_Batch)),
                ("current_row", ctypes.POINTER(ctypes.c_uint8))]


class Slot(ctypes.Structure):
    """One swept parameter: batch, instance, parameter index."""
    _fields_ = [("batch", ctypes.c_uint32), ("inst", ctypes.c_uint32),
                ("param", ctypes.c_uint32)]


class Frozen:
    """A numbered circuit: ``n`` unknowns and one table per device type.

    ``struct()`` returns the C view (``esl_circuit`` / ``orc_circuit``, one
    layout) that stays valid while this object lives.
    """

    def __init__(self, n, batches, current_row, names, where, node_ids):
        self.n = n
        self.batches = [(t, np.ascontiguousarray(nd), np.ascontiguousarray(p))
                        for t, nd, p in batches]
        self.current_row = current_row
        self.names = names
        self.where = where
        self.node_ids = node_ids
        self._c = None

    def struct(self):
        if self._c is None:
            arr = (_Batch * max(1, len(self.batches)))()
            for i, (t, nd, p) in enumerate(self.batches):
                arr[i].type = t
                arr[i].count = nd.shape[0]
                arr[i].nodes = nd.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
                arr[i].params = p.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            c = _Circuit(self.n, len(self.batches), arr,
                         self.current_row.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
            self._c = (c, arr)
        return self._c[0]

    def slot(self, device, param) -> Slot:
        """The sweep slot of ``device``'s ``param`` (card names)."""
        b, i = self.where[device.lower()]
        t = self.batches[b][0]
        return Slot(b, i, PARAM_NAMES[t].index(param.lower()))

    def slots_of(self, type_, param):
        """Every instance of one device type, for per-device variation."""
        out = []
        for b, (t, nd, _) in enumerate(self.batches):
            if t == type_:
                k = PARAM_NAMES[t].index(param)
                out += [Slot(b, i, k) for i in range(nd.shape[0])]
        return out

    def param(self, slot: Slot) -> float:
        return float(self.batches[slot.batch][2][slot.inst, slot.param])

    def unknown(self, name) -> int:
        """Index of a node voltage v(name) or a branch current i(vname)."""
        name = name.lower()
        if name.startswith("v(") and name.endswith(")"):
            return self.node_ids[name[2:-1]]
        if name.startswith("i(") and name.endswith(")"):
            for k, v in self.names.items():
                if v == name:
                    return k
            raise KeyError(name)
        return self.node_ids[name]

    def slots_array(self, slots):
        arr = (Slot * max(1, len(slots)))()
        for i, s in enumerate(slots):
            arr[i] = s
        return arr

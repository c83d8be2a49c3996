"""Test helper: reads the small SPICE decks of the golden fixtures (R, C, V,
I, D, M cards, .model, .dc, .op, .tran, .options, .temp) into a
``espice_b200.circuit.Circuit``. Parsing is not on the sweep-lane path; this
covers only what the committed fixtures use.
"""

from __future__ import annotations

import math
import re

from espice_b200.circuit import Circuit

_SUFFIX = [("meg", 1e6), ("mil", 25.4e-6), ("t", 1e12), ("g", 1e9), ("k", 1e3),
           ("m", 1e-3), ("u", 1e-6), ("n", 1e-9), ("p", 1e-12), ("f", 1e-15)]


def num(tok: str) -> float:
    t = tok.strip().lower()
    m = re.match(r"^([-+]?(?:\d+\.?\d*|\.\d+)(?:e[-+]?\d+)?)([a-z]*)", t)
    if not m:
        raise ValueError(tok)
    v = float(m.group(1))
    rest = m.group(2)
    for s, f in _SUFFIX:
        if rest.startswith(s):
            return v * f
    return v


def _kv(tokens):
    out = {}
    for t in tokens:
        if "=" in t:
            k, v = t.split("=", 1)
            try:
                out[k.lower()] = num(v)
            except ValueError:
                out[k.lower()] = v.lower()
    return out


def _meas(card):
    """A `.meas tran` card of the streamed forms: FIND v AT=t, WHEN v=val
    [RISE|FALL|CROSS=k|LAST] [TD=t], TRIG v VAL=.. .. TARG v VAL=.. .. as
    {"name", "kind", clauses [{"vec", "val", "rise", "fall", "cross", "td",
    "from", "to", "at"}]}."""
    t = re.sub(r"\s*=\s*", "=", card).split()
    assert t[1].lower() == "tran", card
    name, words = t[2].lower(), [w.lower() for w in t[3:]]

    def clause():
        return {"vec": "", "val": 1e99, "rise": -1, "fall": -1, "cross": -1, "td": 0.0, "from": 0.0,
                "to": 0.0, "at": 1e99}

    out = {"name": name, "kind": None, "clauses": []}
    cur = None
    for w in words:
        if w in ("find", "trig", "targ"):
            out["kind"] = out["kind"] or {"find": "find_at", "trig": "trig_targ"}.get(w)
            cur = clause()
            out["clauses"].append(cur)
        elif w == "when":
            out["kind"] = "when"
            cur = clause()
            out["clauses"].append(cur)
        elif "=" in w:
            k, v = w.split("=", 1)
            if k in ("rise", "fall", "cross"):
                cur[k] = -2 if v == "last" else int(num(v))
            elif k in ("val", "td", "from", "to", "at"):
                cur[k] = num(v)
            elif not cur["vec"]:  # WHEN v(x)=level
                cur["vec"], cur["val"] = k, num(v)
        elif not cur["vec"]:
            cur["vec"] = w
    return out


class Deck:
    def __init__(self, text: str):
        self.models = {}
        self.cards = []
        self.analysis = None
        self.options = {}
        self.measures = []
        self.temp = 27.0
        lines = []
        for raw in text.splitlines():
            s = raw.strip()
            if not s or s.startswith("*"):
                continue
            if s.startswith("+") and lines:
                lines[-1] += " " + s[1:]
            else:
                lines.append(s)
        for s in lines:
            s = re.sub(r"\(\s*", "(", s)
            low = s.lower()
            if low.startswith(".model"):
                m = re.match(r"\.model\s+(\S+)\s+(\S+?)\s*\((.*)\)", s, re.I)
                if m:
                    name, kind, body = m.group(1).lower(), m.group(2).lower(), m.group(3)
                else:
                    parts = s.split()
                    name, kind, body = parts[1].lower(), parts[2].lower(), " ".join(parts[3:])
                body = re.sub(r"\s*=\s*", "=", body)
                self.models[name] = (kind, _kv(body.replace(",", " ").split()))
            elif low.startswith(".dc"):
                t = s.split()
                self.analysis = ("dc", t[1].lower(), num(t[2]), num(t[3]), num(t[4]))
                if len(t) >= 9:
                    self.analysis += (t[5].lower(), num(t[6]), num(t[7]), num(t[8]))
            elif low.startswith(".option"):
                body = re.sub(r"\s*=\s*", "=", s)
                self.options.update(_kv(body.split()[1:]))
            elif low.split()[0] == ".op":
                self.analysis = ("op",)
            elif low.startswith(".tran"):
                t = [v for v in s.split() if v.lower() != "uic"]
                tstart = num(t[3]) if len(t) > 3 else 0.0
                tmax = num(t[4]) if len(t) > 4 else 0.0
                self.analysis = ("tran", num(t[1]), num(t[2]), tstart, tmax)
            elif low.startswith(".meas"):
                self.measures.append(_meas(s))
            elif low.startswith(".temp"):
                self.temp = num(s.split()[1])
            elif low.startswith(".end"):
                break
            elif low.startswith("."):
                continue
            else:
                self.cards.append(s)
        if "temp" in self.options:
            self.temp = self.options["temp"]

    def circuit(self) -> Circuit:
        c = Circuit(temp_c=self.temp)
        tnom = self.options.get("tnom", 27.0)
        for s in self.cards:
            t = re.sub(r"\s*=\s*", "=", s).split()
            name = t[0].lower()
            kind = name[0]
            if kind == "r":
                c.R(name, t[1], t[2], num(t[3]))
            elif kind == "c":
                c.C(name, t[1], t[2], num(t[3]))
            elif kind in "vi":
                c_src = c.V if kind == "v" else c.I
                rest = " ".join(t[3:])
                waves = {}
                for w in ("pulse", "sin", "exp", "pwl"):
                    m = re.search(w + r"\s*\(([^)]*)\)", rest, re.I)
                    if m:
                        waves[w] = [num(v) for v in m.group(1).replace(",", " ").split()]
                        rest = rest[: m.start()] + rest[m.end():]
                opts = {}
                toks = []
                for tok in rest.split():
                    if "=" in tok:
                        k, v = tok.split("=", 1)
                        opts[k.lower()] = num(v)
                    else:
                        toks.append(tok)
                dc = None
                if toks and toks[0].lower() == "dc":
                    dc = num(toks[1])
                elif toks:
                    dc = num(toks[0])
                tran = self.analysis and self.analysis[0] == "tran"
                tstep, tstop = (self.analysis[1], self.analysis[2]) if tran else (0.0, 0.0)
                kw = {}
                if "pulse" in waves:
                    pulse = waves["pulse"]
                    if dc is None:
                        dc = pulse[0]
                    if tran:
                        # PULSE defaults from the .tran card (ngspice TRANinit, the
                        # reference's resolvePulseDefaults): TR = TF = TSTEP,
                        # PW = PER = TSTOP
                        full = list(pulse) + [None] * (7 - len(pulse))
                        for k, dflt in ((3, tstep), (4, tstep), (5, tstop), (6, tstop)):
                            if full[k] is None:
                                full[k] = dflt
                        pulse = [0.0 if v is None else v for v in full]
                    kw["pulse"] = pulse
                elif "sin" in waves:
                    sn = waves["sin"] + [0.0] * (6 - len(waves["sin"]))
                    if sn[2] == 0.0 and tran:
                        sn[2] = 1.0 / tstop  # SIN's frequency defaults to 1 / TSTOP
                    if dc is None:
                        dc = sn[0] + sn[1] * math.sin(sn[5] * math.pi / 180.0)
                    kw["sin"] = sn[:6]
                elif "exp" in waves:
                    ex = waves["exp"] + [0.0] * (6 - len(waves["exp"]))
                    if tran:
                        # EXP's omitted (or 0) TD1, TAU1, TAU2 take TSTEP and TD2
                        # TD1 + TSTEP (the reference builder's defaults)
                        if ex[2] == 0.0:
                            ex[2] = tstep
                        if ex[3] == 0.0:
                            ex[3] = tstep
                        if ex[4] == 0.0:
                            ex[4] = ex[2] + tstep
                        if ex[5] == 0.0:
                            ex[5] = tstep
                    if dc is None:
                        dc = ex[0]
                    kw["exp"] = ex[:6]
                elif "pwl" in waves:
                    pts = waves["pwl"]
                    times, values = pts[0::2], pts[1::2]
                    if dc is None:
                        dc = values[0]
                    kw["pwl"] = (times, values, opts.get("r", -1.0), opts.get("td", 0.0))
                c_src(name, t[1], t[2], dc=0.0 if dc is None else dc, **kw)
            elif kind == "d":
                kindm, prm = self.models[t[3].lower()]
                prm = dict(prm)
                prm.setdefault("tnom", tnom)
                area = 1.0
                for tok in t[4:]:
                    if "=" in tok:
                        k, v = tok.split("=")
                        if k.lower() == "area":
                            area = num(v)
                    else:
                        area = num(tok)
                prm.pop("level", None)
                c.D(name, t[1], t[2], area=area, **prm)
            elif kind == "m":
                kindm, prm = self.models[t[5].lower()]
                prm = dict(prm)
                level = prm.pop("level", 1.0)
                if level in (8.0, 49.0):  # BSIM3v3
                    prm.pop("version", None)
                    prm.setdefault("tnom", tnom)
                    prm["type"] = 1.0 if kindm == "nmos" else -1.0
                    prm.update(_kv(t[6:]))
                    c.B3(name, t[1], t[2], t[3], t[4], **prm)
                    continue
                prm.setdefault("tnom", tnom)
                prm["type"] = 1.0 if kindm == "nmos" else -1.0
                prm.update(_kv(t[6:]))
                c.M(name, t[1], t[2], t[3], t[4], **prm)
            else:
                raise ValueError(f"card {s!r} is not supported")
        return c

    def newton_opts(self):
        return dict(reltol=self.options.get("reltol", 1e-3),
                    abstol=self.options.get("abstol", 1e-12),
                    vntol=self.options.get("vntol", 1e-6))


def sweep_values(start, stop, step):
    """ngspice's accumulated sweep axis (v += step), as dc.zig steps it."""
    import math
    if step == 0 or (stop - start) * math.copysign(1.0, step) < 0:
        n = 1
    else:
        n = int(math.floor((stop - start) / step + 1e-6)) + 1
    out = []
    v = start
    for _ in range(n):
        out.append(v)
        v += step
    return out

"""The oracle's BSIM3v3 DC core: its dual-number Jacobian against central
finite differences of its own residuals (the reference checks its device
Jacobians against finite differences at rtol 1e-5,
src/device/tests/jacobian_fd.zig:144), over bias points in every operating
region of the card variants the GPU tests use. Its values are pinned
against ngspice by the golden fixtures (test_oracle_golden.py)."""

import ctypes

import numpy as np
import pytest

from espice_b200 import decks
from espice_b200.circuit import B3, B3_DEFAULTS, B3_PARAMS
from oracle import oracle

f64p = ctypes.POINTER(ctypes.c_double)


def _params(card, temp_c=27.0, **inst):
    kw = dict(B3_DEFAULTS, temp=temp_c + 273.15, l=0.18e-6, w=2e-6)
    kw.update(card)
    kw.update(inst)
    return np.array([kw[p] for p in B3_PARAMS], dtype=np.float64)


def _stamp(prm, x):
    f = np.zeros(6)
    J = np.zeros(36)
    rc = oracle.lib().orc_dev_stamp(ctypes.c_uint32(B3), prm.ctypes.data_as(f64p), x.ctypes.data_as(f64p),
                                    f.ctypes.data_as(f64p), J.ctypes.data_as(f64p))
    assert rc == 0
    return f, J.reshape(6, 6)


CARDS = [("nmos_fixture", decks.B3_NMOS[0]), ("nmos_derived_rsh_isub", decks.B3_NMOS[1]),
         ("nmos_mobmod3", decks.B3_NMOS[2]), ("pmos_fixture", decks.B3_PMOS)]


def test_parameter_slots_match_the_oracle():
    assert len(B3_PARAMS) == oracle.lib().orc_params_per(B3) == 109
    assert oracle.lib().orc_nodes_per(B3) == 6


@pytest.mark.parametrize("name,card", CARDS)
@pytest.mark.parametrize("temp_c", [27.0, 85.0])
def test_jacobian_matches_finite_differences(name, card, temp_c):
    prm = _params(card, temp_c)
    rng = np.random.default_rng(11)
    t = card["type"]
    checked = 0
    for _ in range(200):
        # nodes d g s b di si; type-frame biases spanning cut-off,
        # subthreshold, linear and saturation, both channel directions and
        # forward and reverse body bias
        vs = rng.uniform(-0.2, 0.2)
        vgs, vds, vbs = rng.uniform(-0.3, 1.8), rng.uniform(-1.8, 1.8), rng.uniform(-1.5, 0.4)
        x = np.empty(6)
        x[2] = x[5] = vs
        x[1] = vs + t * vgs
        x[0] = x[4] = vs + t * vds
        x[3] = vs + t * vbs
        if prm[B3_PARAMS.index("rsh")] > 0:
            x[4] = x[0] - t * 0.01 * np.sign(vds)
            x[5] = x[2] + t * 0.01 * np.sign(vds)
        f0, J = _stamp(prm, x)
        fd = np.zeros((6, 6))
        for k in range(6):
            h = 1e-6 * max(1.0, abs(x[k]))
            xp, xm = x.copy(), x.copy()
            xp[k] += h
            xm[k] -= h
            fd[:, k] = (_stamp(prm, xp)[0] - _stamp(prm, xm)[0]) / (2 * h)
        scale = np.abs(J).max(axis=1, keepdims=True) + 1e-15
        err = np.abs(J - fd) / (1e-5 * scale + 1e-5 * np.abs(J))
        assert np.all(err <= 1.0), (name, vgs, vds, vbs, float(err.max()), J, fd)
        checked += 1
    assert checked == 200

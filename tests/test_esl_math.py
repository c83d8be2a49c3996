"""The exp, log and pow that the device models and the oracle share
(espice_b200/csrc/esl_math.h), checked on the CPU (through the oracle build):
- accuracy: within 2 ulp of the correctly rounded value on exp and log over
  their whole ranges (the reference value from Python's decimal module at 40
  digits), and pow within 2 |y ln x| + 3 ulp on the models' argument ranges;
- special values as C's exp, log and pow return them;
- what replacing the C library's functions changes: the oracle built with
  glibc's exp, log and pow and the oracle built with the shared ones take the
  same Newton iteration counts on every lane of the synthetic DC decks and the
  reference's DC fixtures, and their solutions differ only in the last bits.
"""

import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

from espice_b200 import decks
from oracle import oracle

getcontext().prec = 40


def _ulp(x):
    return math.ulp(x) if x != 0 else 5e-324


def _ref(fn, xs, ys=None):
    out = []
    for i, x in enumerate(xs):
        d = Decimal(float(x))
        if fn == "exp":
            out.append(float(d.exp()))
        elif fn == "log":
            out.append(float(d.ln()))
        else:
            out.append(float((Decimal(float(ys[i])) * d.ln()).exp()))
    return np.array(out)


def test_exp_accuracy():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-745, 709.78, 3000), rng.uniform(-40, 40, 3000), rng.uniform(-1e-3, 1e-3, 500)])
    got = oracle.math("exp", xs)
    ref = _ref("exp", xs)
    err = np.abs(got - ref) / np.array([_ulp(r) for r in ref])
    assert err.max() <= 2.0, (float(err.max()), float(xs[np.argmax(err)]))


def test_log_accuracy():
    rng = np.random.default_rng(2)
    xs = np.concatenate([np.ldexp(rng.uniform(1, 2, 3000), rng.integers(-1074, 1023, 3000)),
                         rng.uniform(0.5, 2.0, 3000), 1 + rng.uniform(-1e-6, 1e-6, 500)])
    xs = xs[xs > 0]
    got = oracle.math("log", xs)
    ref = _ref("log", xs)
    err = np.abs(got - ref) / np.array([_ulp(r) for r in ref])
    assert err.max() <= 2.0, (float(err.max()), float(xs[np.argmax(err)]))


def test_pow_accuracy():
    rng = np.random.default_rng(3)
    xs = rng.uniform(0.01, 3.0, 2000)
    ys = rng.uniform(-3.0, 3.0, 2000)
    got = oracle.math("pow", xs, ys)
    ref = _ref("pow", xs, ys)
    bound = 2.0 * np.abs(ys * np.log(xs)) + 3.0
    err = np.abs(got - ref) / np.array([_ulp(r) for r in ref])
    assert (err <= bound).all(), float((err / bound).max())


def test_special_values():
    inf, nan = math.inf, math.nan
    e = oracle.math("exp", [0.0, nan, inf, -inf, 710.0, -746.0, 1.0])
    assert e[0] == 1.0 and np.isnan(e[1]) and e[2] == inf and e[3] == 0.0 and e[4] == inf and e[5] == 0.0
    assert abs(e[6] - math.e) <= _ulp(math.e)
    lg = oracle.math("log", [1.0, 0.0, -1.0, inf, nan, 5e-324])
    assert lg[0] == 0.0 and lg[1] == -inf and np.isnan(lg[2]) and lg[3] == inf and np.isnan(lg[4])
    assert abs(lg[5] - math.log(5e-324)) <= 2 * _ulp(math.log(5e-324))
    p = oracle.math("pow", [-2.0, 0.0, 0.0, -8.0, 3.0, 1.0, -2.0], [3.0, -1.0, 2.0, 1 / 3, 0.0, nan, 2.0])
    assert p[0] == -8.0 and p[1] == inf and p[2] == 0.0 and np.isnan(p[3]) and p[4] == 1.0 and p[5] == 1.0
    assert p[6] == 4.0


def test_exp_exact_powers_and_log_of_powers():
    ks = np.arange(-1000, 1001, 37).astype(np.float64)
    assert np.array_equal(oracle.math("log", np.ldexp(1.0, ks.astype(int))), ks * math.log(2)) or \
        np.all(np.abs(oracle.math("log", np.ldexp(1.0, ks.astype(int))) - ks * math.log(2))
               <= 2 * np.array([_ulp(v) for v in ks * math.log(2)]))


@pytest.mark.parametrize("deck,seed", [("grid", 1), ("grid", 2), ("bsim3", 1)])
def test_libm_and_shared_transcendentals_agree_on_lanes(deck, seed):
    if deck == "grid":
        fr, slots, values = decks.grid_diodes(seed=seed, points=256)
        warm = np.zeros(fr.n)
    else:
        fr, slots, values = decks.bsim3_inverters(seed=seed, lanes=128)
        warm = None
    xa, ia, ca, _ = oracle.dc_points_trace(fr, slots, values, warm=warm)
    xb, ib, cb, _ = oracle.dc_points_trace(fr, slots, values, warm=warm, libm=True)
    assert np.array_equal(ca, cb)
    assert np.array_equal(ia, ib), np.flatnonzero(ia != ib)
    assert np.all(np.abs(xa - xb) <= 1e-12 + 1e-12 * np.abs(xa))

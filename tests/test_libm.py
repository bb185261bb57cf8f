"""Accuracy of the project's log/exp/pow (trinity_b200/csrc/trn_libm.h)
against the platform libm, on random and edge inputs. These functions replace
libm on every side that must agree bit for bit (kernels, oracle, pinned
reference build); bounds: log and exp within 2 ulp, pow(x, -1/6) within
8 ulp (it goes through exp(y log x)), pow(x, 2) and pow(x, 3) exactly x*x and
(x*x)*x."""
import math

import numpy as np

from tests.oracle_lib import lib


def ulp_err(got, want):
    return abs(got - want) / math.ulp(want) if want != 0 else abs(got)


def test_log_accuracy():
    L = lib()
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.exp(rng.uniform(-700, 700, 20000)), rng.uniform(0.5, 2.0, 20000),
                         [1.0, 2.0, 0.5, 6.25, 1e18, 1e-300, 5e-324, 1.7976931348623157e308]])
    worst = max(ulp_err(L.orc_log_fn(float(x)), math.log(x)) for x in xs if math.log(x) != 0)
    assert worst <= 2.0, worst
    assert L.orc_log_fn(1.0) == 0.0
    assert math.isinf(L.orc_log_fn(0.0)) and L.orc_log_fn(0.0) < 0
    assert math.isnan(L.orc_log_fn(-1.0))


def test_exp_accuracy():
    L = lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-700, 700, 20000), rng.uniform(-1, 1, 20000), [0.0, 1.0, -1.0, 41.4]])
    worst = max(ulp_err(L.orc_exp_fn(float(x)), math.exp(x)) for x in xs)
    assert worst <= 2.0, worst
    assert L.orc_exp_fn(0.0) == 1.0
    assert math.isinf(L.orc_exp_fn(800.0)) and L.orc_exp_fn(-800.0) == 0.0


def test_pow_paths():
    L = lib()
    rng = np.random.default_rng(2)
    for x in rng.uniform(-1e3, 1e3, 2000):
        x = float(x)
        assert L.orc_pow_fn(x, 2.0) == x * x
        assert L.orc_pow_fn(x, 3.0) == (x * x) * x
    worst = 0.0
    for x in np.exp(rng.uniform(-45, 45, 20000)):
        x = float(x)
        worst = max(worst, ulp_err(L.orc_pow_fn(x, -1.0 / 6.0), x ** (-1.0 / 6.0)))
    assert worst <= 8.0, worst

"""The reproducible transcendental functions (delta_ray_b200/csrc/dr_math.h).

The renderer evaluates sin, cos, atan, atan2, acos, exp, log and pow with its
own routines so that the GPU and the oracle's CPU build round them to the same
float.  Here, compiled for the CPU, they are checked against numpy's
double-precision functions rounded to float: sin, cos, exp, log and pow
(evaluated in double) at most one float ulp apart and equal on all but a
vanishing share of inputs; atan, atan2 and acos (evaluated in float) within 3
ulp.  The GPU
test (test_dr_math_gpu.py) checks that the device build gives the same bits.
"""
import numpy as np
import pytest

from native import harness


FLOAT_EVALUATED = ("atan", "atan2", "acos")


def ulp_distance(a, b):
    """Distance in float32 units in the last place (NaNs must match)."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    both_nan = np.isnan(a) & np.isnan(b)
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    d = np.abs(ia - ib)
    d[both_nan] = 0
    d[np.isnan(a) ^ np.isnan(b)] = 1 << 40
    return d


def math_inputs(seed=0):
    """Inputs per function: dense grids over the ranges the renderer uses and
    log-uniform samples beyond them, with the special values."""
    rng = np.random.default_rng(seed)
    n = 200_000

    def logu(lo, hi, k):
        return np.exp(rng.uniform(np.log(lo), np.log(hi), k))

    ang = np.concatenate([rng.uniform(-8, 8, n), np.linspace(-2 * np.pi, 2 * np.pi, 20001),
                          logu(1e-30, 1e4, n // 4) * rng.choice([-1, 1], n // 4), [0.0, -0.0, np.pi, -np.pi]])
    ratio = np.concatenate([logu(1e-38, 1e38, n) * rng.choice([-1, 1], n), rng.uniform(-2, 2, n),
                            [0.0, -0.0, 1.0, -1.0, np.inf, -np.inf]])
    unit = np.concatenate([rng.uniform(-1, 1, n), 1 - logu(1e-8, 1, n // 4), -1 + logu(1e-8, 1, n // 4),
                           [1.0, -1.0, 0.0, -0.0]])
    ex = np.concatenate([rng.uniform(-110, 89, n), rng.uniform(-1, 1, n // 4), [0.0, -0.0, 88.7, -103.9]])
    lg = np.concatenate([logu(1e-45, 3e38, n), rng.uniform(0.5, 2, n // 4), [1.0, 2.0, 1e-45, 3.4e38]])
    px = np.concatenate([rng.uniform(0, 1, n), logu(1e-3, 10, n // 2), [0.0, 1.0, 0.5, 2.0]])
    py = np.concatenate([logu(1, 2000, n), rng.uniform(-5, 5, n // 2), [3.0, 0.0, 5.0, -2.0]])
    yx = rng.normal(size=(2, n)) * logu(1e-3, 1e3, n)
    yx = np.concatenate([yx, [[0.0, 0.0, -0.0, 1.0, -1.0, 0.0, np.inf], [1.0, -1.0, -1.0, 0.0, 0.0, 0.0, np.inf]]], 1)
    f = lambda a: np.asarray(a, np.float32)  # noqa: E731
    return {
        "sin": (f(ang), None), "cos": (f(ang), None), "atan": (f(ratio), None), "acos": (f(unit), None),
        "exp": (f(ex), None), "log": (f(lg), None), "pow": (f(px), f(py)), "atan2": (f(yx[0]), f(yx[1])),
    }


def numpy_reference(name, x, y):
    x64 = x.astype(np.float64)
    y64 = None if y is None else y.astype(np.float64)
    with np.errstate(all="ignore"):
        r = {"sin": lambda: np.sin(x64), "cos": lambda: np.cos(x64), "atan": lambda: np.arctan(x64),
             "acos": lambda: np.arccos(x64), "exp": lambda: np.exp(x64), "log": lambda: np.log(x64),
             "pow": lambda: np.power(x64, y64), "atan2": lambda: np.arctan2(x64, y64)}[name]()
        return r.astype(np.float32)


@pytest.mark.parametrize("name", sorted(harness.MATH_FUNCS))
def test_reproducible_math_is_within_one_ulp_of_double_precision(name):
    x, y = math_inputs()[name]
    got = harness.math_eval(name, x, y)
    ref = numpy_reference(name, x, y)
    d = ulp_distance(got, ref)
    worst = (name, x[d.argmax()], None if y is None else y[d.argmax()], got[d.argmax()], ref[d.argmax()])
    if name in FLOAT_EVALUATED:
        # evaluated in float: a few ulp, most results the nearest float
        assert d.max() <= 3, worst
        assert (d == 0).mean() >= 0.7, (name, (d != 0).mean())
    else:
        # evaluated in double and rounded once: the nearest float but for
        # values within ~1e-15 of a rounding boundary
        assert d.max() <= 1, worst
        assert (d == 0).mean() >= 0.9999, (name, (d != 0).sum())


def test_reproducible_math_special_values():
    f = harness.math_eval
    assert f("acos", np.array([1.0, -1.0], np.float32))[0] == 0.0
    assert f("acos", np.array([-1.0], np.float32))[0] == np.float32(np.pi)
    assert np.isnan(f("acos", np.array([1.5], np.float32))[0])
    assert np.isnan(f("log", np.array([-1.0], np.float32))[0])
    assert f("log", np.array([0.0], np.float32))[0] == -np.inf
    assert f("exp", np.array([-200.0], np.float32))[0] == 0.0
    assert f("exp", np.array([100.0], np.float32))[0] == np.inf
    assert f("pow", np.array([0.0], np.float32), np.array([2.0], np.float32))[0] == 0.0
    assert f("pow", np.array([-2.0], np.float32), np.array([3.0], np.float32))[0] == -8.0
    assert np.isnan(f("pow", np.array([-2.0], np.float32), np.array([0.5], np.float32))[0])
    a2 = f("atan2", np.array([0.0, -0.0, 0.0], np.float32), np.array([-1.0, -1.0, 1.0], np.float32))
    assert a2[0] == np.float32(np.pi) and a2[1] == -np.float32(np.pi) and a2[2] == 0.0

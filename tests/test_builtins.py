"""Accuracy of the shared single-precision WGSL built-ins (wgsl_builtins.h) against float64,
evaluated through the oracle library (the same header is compiled into the kernels)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle

OPS = {"sin": 0, "cos": 1, "exp": 2, "log": 3, "exp2": 4, "log2": 5, "atan2": 6, "asin": 7, "acos": 8, "pow": 9}


def ulp_error(got: np.ndarray, ref: np.ndarray) -> np.ndarray:
    ref32 = ref.astype(np.float32)
    return np.abs(got.astype(np.float64) - ref) / np.abs(np.spacing(ref32)).astype(np.float64)


@pytest.mark.parametrize("name,lo,hi,fn,bound", [
    ("sin", -40.0, 40.0, np.sin, 2.0), ("cos", -40.0, 40.0, np.cos, 2.0), ("exp", -87.0, 88.0, np.exp, 2.0),
    ("exp2", -125.0, 127.0, np.exp2, 2.0), ("asin", -1.0, 1.0, np.arcsin, 4.0), ("acos", -1.0, 1.0, np.arccos, 4.0),
])
def test_unary_accuracy(name, lo, hi, fn, bound):
    x = np.random.default_rng(1).uniform(lo, hi, 200_000).astype(np.float32)
    got = oracle.builtin(OPS[name], x)
    assert ulp_error(got, fn(x.astype(np.float64))).max() <= bound


@pytest.mark.parametrize("name,fn", [("log", np.log), ("log2", np.log2)])
def test_log_accuracy(name, fn):
    x = np.exp(np.random.default_rng(2).uniform(-85, 85, 200_000)).astype(np.float32)
    x = np.concatenate([x, np.float32([1e-40, 3e-45, 1.0, 2.0, 0.5])])   # subnormals, exact points
    got = oracle.builtin(OPS[name], x)
    assert ulp_error(got, fn(x.astype(np.float64))).max() <= 3.0


def test_atan2_accuracy_and_quadrants():
    rng = np.random.default_rng(3)
    y = rng.normal(size=200_000).astype(np.float32)
    x = rng.normal(size=200_000).astype(np.float32)
    got = oracle.builtin(OPS["atan2"], y, x)
    assert ulp_error(got, np.arctan2(y.astype(np.float64), x.astype(np.float64))).max() <= 3.0
    sp = oracle.builtin(OPS["atan2"], np.float32([0, -0.0, 0, 1, -1, 1]), np.float32([1, 1, -1, 0, 0, np.inf]))
    np.testing.assert_array_equal(sp, np.float32([0, -0.0, np.pi, np.pi / 2, -np.pi / 2, 0]))


def test_pow_follows_exp2_log2_definition():
    """WGSL defines pow(x, y) as exp2(y * log2(x)): relative error grows with |y log2 x|."""
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 4, 100_000).astype(np.float32)
    y = rng.uniform(0, 5, 100_000).astype(np.float32)
    got = oracle.builtin(OPS["pow"], x, y).astype(np.float64)
    ref = np.power(x.astype(np.float64), y.astype(np.float64))
    rel = np.abs(got - ref) / np.maximum(ref, 1e-30)
    assert rel.max() < 5e-6
    sp = oracle.builtin(OPS["pow"], np.float32([0, 0, 1, 2]), np.float32([5, 0.4545, 3, 0.5]))
    np.testing.assert_allclose(sp, [0, 0, 1, np.sqrt(2)], rtol=1e-6)


def test_special_values():
    e = oracle.builtin(OPS["exp"], np.float32([0, -200, 100, np.nan, np.inf, -np.inf]))
    assert e[0] == 1 and e[1] == 0 and np.isinf(e[2]) and np.isnan(e[3]) and np.isinf(e[4]) and e[5] == 0
    l = oracle.builtin(OPS["log"], np.float32([0, -1, np.inf, np.nan, 1]))
    assert np.isneginf(l[0]) and np.isnan(l[1]) and np.isinf(l[2]) and np.isnan(l[3]) and l[4] == 0

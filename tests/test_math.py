"""The shared intrinsics (aviatorengine2_b200/csrc/ae_math.h) against libm in
double: sin/cos/tan/exp/log/pow/atan2/acos within stated ulp bounds.  These
are the definitions the kernels, the oracle and the reference pin all use."""
import ctypes

import numpy as np
import pytest

import _oracle as O


def run(fn, x, y=None):
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros_like(x) if y is None else np.ascontiguousarray(y, np.float32)
    out = np.zeros_like(x)
    O.oracle().oracle_math(ctypes.c_int(fn), O.ptr(x), O.ptr(y), O.ptr(out), ctypes.c_uint32(len(x)))
    return out


def ulp_err(got, want):
    want32 = want.astype(np.float32)
    spacing = np.spacing(np.abs(want32).astype(np.float32)).astype(np.float64)
    spacing = np.maximum(spacing, np.finfo(np.float32).tiny)
    return np.abs(got.astype(np.float64) - want) / spacing


rng = np.random.default_rng(7)


@pytest.mark.parametrize("fn,ref,lo,hi,bound", [
    (0, np.sin, -100.0, 100.0, 2.0),
    (1, np.cos, -100.0, 100.0, 2.0),
    (2, np.tan, -1.5, 1.5, 4.0),
    (3, np.exp, -80.0, 80.0, 2.0),
    (4, np.log, 1e-30, 1e30, 2.0),
    (7, np.arccos, -1.0, 1.0, 6.0),
])
def test_unary_within_ulps(fn, ref, lo, hi, bound):
    if fn == 4:
        x = np.exp(rng.uniform(np.log(lo), np.log(hi), 200000)).astype(np.float32)
    else:
        x = rng.uniform(lo, hi, 200000).astype(np.float32)
    got = run(fn, x)
    want = ref(x.astype(np.float64))
    if fn in (0, 1):
        # absolute error near zeros of the function, relative elsewhere
        err = np.abs(got.astype(np.float64) - want)
        assert err.max() < bound * 6e-8
    else:
        assert ulp_err(got, want).max() <= bound


def test_sin_cos_angle_range_of_random_direction():
    # RandomDirection draws a in [0, 2 pi) (hybrid:245-251).
    a = rng.uniform(0, 6.2831853, 200000).astype(np.float32)
    for fn, ref in ((0, np.sin), (1, np.cos)):
        err = np.abs(run(fn, a).astype(np.float64) - ref(a.astype(np.float64)))
        assert err.max() < 1.2e-7


def test_pow_integer_and_fractional():
    x = rng.uniform(0.0, 1.0, 100000).astype(np.float32)
    assert np.array_equal(run(5, x, np.full_like(x, 2.0)), (x * x).astype(np.float32))
    got = run(5, x, np.full_like(x, 1.0 / 2.4))
    want = np.power(x.astype(np.float64), np.float64(np.float32(1.0 / 2.4)))
    assert ulp_err(got[x > 1e-3], want[x > 1e-3]).max() <= 8


def test_atan2_quadrants():
    y = rng.uniform(-10, 10, 100000).astype(np.float32)
    x = rng.uniform(-10, 10, 100000).astype(np.float32)
    got = run(6, y, x)
    assert np.abs(got.astype(np.float64) - np.arctan2(y.astype(np.float64), x.astype(np.float64))).max() < 5e-7


def test_rng_matches_reference_hash():
    # hybrid:238-243, evaluated in numpy uint32 arithmetic.
    seeds = rng.integers(0, 2 ** 32, 10000, dtype=np.uint64).astype(np.uint32)
    got = run(8, seeds.view(np.float32))
    s = (seeds.astype(np.uint64) * 747796405 + 2891336453) & 0xFFFFFFFF
    x = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
    v = ((x >> 22) ^ x).astype(np.uint32)
    want = (v.astype(np.float32) / np.float32(4294967296.0)).astype(np.float32)
    assert np.array_equal(got, want)

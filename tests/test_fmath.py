"""The portable transcendentals (csrc/fmath.h) against float64 references:
a few ulp for sin/cos/acos/atan2/exp/log/log2; pow's error grows with
|y log2 x| as exp2(y log2 x) does."""
from __future__ import annotations

import numpy as np
import pytest


def ulp_err(got: np.ndarray, ref: np.ndarray) -> np.ndarray:
    r32 = ref.astype(np.float32)
    sp = np.spacing(np.abs(r32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - ref) / sp


CASES = {
    0: (lambda r: r.uniform(-20, 20, 200000), None, np.sin, 3.0),
    1: (lambda r: r.uniform(-20, 20, 200000), None, np.cos, 3.0),
    2: (lambda r: np.concatenate([r.uniform(-1, 1, 150000), 1 - r.uniform(0, 1e-3, 50000)]), None, np.arccos, 4.0),
    4: (lambda r: r.uniform(-87, 88, 200000), None, np.exp, 3.0),
    5: (lambda r: np.exp(r.uniform(-85, 85, 200000)), None, np.log, 3.0),
    6: (lambda r: np.exp(r.uniform(-85, 85, 200000)), None, np.log2, 4.0),
}


@pytest.mark.parametrize("op", sorted(CASES))
def test_unary_accuracy(oracle, op):
    gen, _, ref, tol = CASES[op]
    rng = np.random.default_rng(op + 100)
    a = gen(rng).astype(np.float32)
    got = oracle.math(op, a, libm=False)
    want = ref(a.astype(np.float64))
    # Around zeros of sin/cos the ulp measure blows up: use absolute error.
    small = np.abs(want) < 1e-3
    assert np.max(ulp_err(got[~small], want[~small])) <= tol
    if small.any():
        assert np.max(np.abs(got[small] - want[small])) <= 1e-9


def test_atan2_accuracy_and_quadrants(oracle):
    rng = np.random.default_rng(7)
    y = rng.standard_normal(200000).astype(np.float32)
    x = rng.standard_normal(200000).astype(np.float32)
    got = oracle.math(3, y, x)
    want = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    assert np.max(ulp_err(got, want)) <= 4.0
    sp = np.array([0.0, -0.0, 0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, 1.0], np.float32)
    sx = np.array([1.0, 1.0, -1.0, -1.0, 0.0, 0.0, 1.0, -np.inf, np.inf], np.float32)
    got = oracle.math(3, sp, sx)
    want = np.arctan2(sp, sx).astype(np.float32)
    assert np.array_equal(np.signbit(got), np.signbit(want))
    assert np.allclose(got, want, rtol=2e-7, atol=0)


def test_pow_accuracy_in_the_tracers_ranges(oracle):
    rng = np.random.default_rng(9)
    # resolve.wgsl sRGB curves.
    x = rng.uniform(0.0031308, 1.0, 100000).astype(np.float32)
    g = oracle.math(7, x, np.full_like(x, 1 / 2.4))
    assert np.max(ulp_err(g, x.astype(np.float64) ** np.float64(np.float32(1 / 2.4)))) <= 6
    c = rng.uniform(0.04045, 1.0, 100000).astype(np.float32)
    b = ((c + np.float32(0.055)) / np.float32(1.055)).astype(np.float32)
    g = oracle.math(7, b, np.full_like(b, 2.4))
    assert np.max(ulp_err(g, b.astype(np.float64) ** np.float64(np.float32(2.4)))) <= 16
    # d_charlie: pow(sin^2, 1/(2 alpha)), relative error bounded by |y log2 x| ulp.
    s2 = rng.uniform(0.01, 1.0, 100000).astype(np.float32)
    e = rng.uniform(0.5, 50.0, 100000).astype(np.float32)
    g = oracle.math(7, s2, e)
    want = s2.astype(np.float64) ** e.astype(np.float64)
    ok = want > 1e-30
    bound = 8 + 4 * np.abs(e.astype(np.float64) * np.log2(s2.astype(np.float64)))
    assert np.all(ulp_err(g[ok], want[ok]) <= bound[ok])


def test_special_values(oracle):
    nan = np.float32(np.nan)
    assert np.isnan(oracle.math(0, np.array([np.inf, nan], np.float32))).all()
    assert np.isnan(oracle.math(2, np.array([1.5, -1.0000001], np.float32))).all()
    assert oracle.math(2, np.array([-1.0], np.float32))[0] == np.float32(np.pi)
    assert oracle.math(4, np.array([-200.0, 100.0], np.float32)).tolist() == [0.0, np.inf]
    assert oracle.math(5, np.array([0.0, -1.0], np.float32))[0] == -np.inf
    assert np.isnan(oracle.math(5, np.array([-1.0], np.float32)))[0]
    one = np.ones(3, np.float32)
    assert oracle.math(7, np.array([1.0, 0.0, 2.0], np.float32), np.array([7.0, 3.0, 0.0], np.float32)).tolist() == [
        1.0, 0.0, 1.0]
    # Subnormal input to log2.
    assert oracle.math(6, np.array([2.0 ** -140], np.float32))[0] == -140.0
    assert one.sum() == 3


def test_libm_and_portable_agree_to_a_few_ulp(oracle):
    rng = np.random.default_rng(1)
    a = rng.uniform(-3, 3, 100000).astype(np.float32)
    for op in (0, 1):
        p, l = oracle.math(op, a, libm=False), oracle.math(op, a, libm=True)
        assert np.max(ulp_err(p[np.abs(l) > 1e-3], l[np.abs(l) > 1e-3].astype(np.float64))) <= 4

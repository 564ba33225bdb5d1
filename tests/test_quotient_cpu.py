"""The FP32 velocity of the cell update, u = m / r, is computed as one correctly rounded reciprocal
y = RN(1/r) shared by the components, q = RN(m y), and Markstein's correction RN(q + RN(m - r q) y)
with fused multiply-adds (aa_step.cuh, update_cell). This checks, in exact rational arithmetic,
that the corrected quotient equals the correctly rounded quotient RN(m / r) over the values the
kernels see (densities near 1, momenta up to a few tenths, both signs) and over extreme
significands, so the kernels' results are those of an IEEE division. No GPU needed."""

from __future__ import annotations

from fractions import Fraction

import numpy as np


def rn32(x: Fraction) -> Fraction:
    """x rounded to the nearest float32 (ties to even); normal range."""
    if x == 0:
        return Fraction(0)
    sign = -1 if x < 0 else 1
    a = abs(x)
    e = a.numerator.bit_length() - a.denominator.bit_length()
    while Fraction(2) ** e > a:
        e -= 1
    while Fraction(2) ** (e + 1) <= a:
        e += 1
    ulp = Fraction(2) ** (e - 23)
    q, rem = divmod(a, ulp)
    if 2 * rem > ulp or (2 * rem == ulp and q % 2 == 1):
        q += 1
    return sign * q * ulp


def corrected_quotient(m: Fraction, r: Fraction) -> Fraction:
    y = rn32(1 / r)
    q = rn32(m * y)
    e = rn32(m - r * q)  # fused: m - r q exact, one rounding
    return rn32(e * y + q)  # fused


def _f(v) -> Fraction:
    return Fraction(float(np.float32(v)))


def test_corrected_quotient_is_correctly_rounded():
    rng = np.random.default_rng(7)
    r = 1.0 + rng.uniform(-0.05, 0.05, 3000)
    r = np.concatenate([r, rng.uniform(0.5, 2.0, 1000), 1.0 + rng.integers(-4096, 4096, 500) * 2.0**-23])
    m = rng.uniform(-0.3, 0.3, r.size) * 10.0 ** rng.integers(-6, 1, r.size)
    # extreme significands: all ones, just above powers of two
    m[:64] = [(2 - 2.0**-23) * 2.0 ** -k for k in range(1, 65)][:64]
    r[:64] = [1 + 2.0**-23 * (k + 1) for k in range(64)]
    bad = []
    for mi, ri in zip(m, r):
        fm, fr = _f(mi), _f(ri)
        if fm == 0:
            continue
        if corrected_quotient(fm, fr) != rn32(fm / fr):
            bad.append((float(fm), float(fr)))
    assert not bad, bad[:5]


def test_uncorrected_product_is_not_always_the_quotient():
    # the plain m * (1/r) differs from the quotient in a share of cases near r = 1 (why the
    # correction is there)
    rng = np.random.default_rng(3)
    diff = 0
    for _ in range(2000):
        fm, fr = _f(rng.uniform(-0.1, 0.1)), _f(1 + rng.uniform(-0.01, 0.01))
        diff += rn32(fm * rn32(1 / fr)) != rn32(fm / fr)
    assert diff > 0

"""CPU check of the division method of the Thomas forward sweeps (csrc/div_rn.cuh).

The kernels form y = RN(1/D) off the recurrence's chain and then, per quotient,
q = RN(u y), r = RN(u - D q) (one fused multiply-add, exact here), and return q when
r == 0, else RN(q + r y) (a second fused multiply-add): Markstein's final correction step.
Here every rounding is restated with exact rationals (a fused multiply-add is one rounding
of the exact value; Python rounds int / int and float / float correctly), and the result is
compared with the correctly rounded quotient u / D bit for bit, signs of zero included.
The GPU test (test_gpu_division.py) runs the same comparison against __ddiv_rn."""
import math
import random
import struct
from fractions import Fraction

import pytest


def rn(x: Fraction) -> float:
    """Round an exact rational to the nearest double (ties to even)."""
    return x.numerator / x.denominator


def fma(a: float, b: float, c: float) -> float:
    """RN(a b + c) with one rounding; an exact zero gets IEEE 754's round-to-nearest sign."""
    exact = Fraction(a) * Fraction(b) + Fraction(c)
    if exact != 0:
        return rn(exact)
    if (a == 0 or b == 0) and c == 0:
        # zero plus zero: -0 only when both are -0 (the product's sign is sign(a) sign(b))
        prod_neg = math.copysign(1.0, a) * math.copysign(1.0, b) < 0
        return -0.0 if prod_neg and math.copysign(1.0, c) < 0 else 0.0
    return 0.0  # x + (-x) with x nonzero


def ieee_div(u: float, D: float) -> float:
    """RN(u / D) with IEEE 754's signed zeros and infinities (D is never zero here)."""
    if math.isinf(u) or math.isnan(u):
        return u / D if not math.isnan(u) else math.nan
    return u / D


def div_by_recip(u: float, D: float) -> float:
    """The kernels' division for a pivot 2^-40 <= |D| <= 2^1000: the correction step when
    2^-900 <= |q| < 2^1000 (or u = 0), else IEEE division."""
    assert 2.0 ** -40 <= abs(D) <= 2.0 ** 1000
    y = 1.0 / D  # RN(1/D), as __drcp_rn
    q = u * y  # RN(u y)
    if u != 0.0 and not (2.0 ** -900 <= abs(q) < 2.0 ** 1000):
        return ieee_div(u, D)
    r = fma(-D, q, u)
    return q if r == 0.0 else fma(r, y, q)


def correction_step(u: float, D: float) -> float:
    """The correction step alone (no window), to show where it stops being exact."""
    y = 1.0 / D
    q = u * y
    r = fma(-D, q, u)
    return q if r == 0.0 else fma(r, y, q)


def bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", x))[0]


def random_double(rng: random.Random, span: int) -> float:
    mant = rng.getrandbits(52)
    sel = rng.randrange(8)
    if sel == 0:
        mant = (1 << 52) - 1
    elif sel == 1:
        mant = 0
    ex = 1023 + rng.randrange(-span, span + 1)
    sign = rng.getrandbits(1)
    return struct.unpack("<d", struct.pack("<Q", (sign << 63) | (ex << 52) | mant))[0]


@pytest.mark.parametrize("seed", [11, 12])
def test_correction_step_gives_the_correctly_rounded_quotient(seed):
    rng = random.Random(seed)
    for _ in range(20000):
        u = random_double(rng, 200)
        D = random_double(rng, 40)
        assert bits(div_by_recip(u, D)) == bits(u / D), (u, D)


@pytest.mark.parametrize("u", [0.0, -0.0])
@pytest.mark.parametrize("D", [3.0, -3.0, 648.5296676163562, -1e-3])
def test_zero_numerator_keeps_the_quotient_sign(u, D):
    assert bits(div_by_recip(u, D)) == bits(u / D)


def test_exact_quotients_take_the_product():
    # r == 0 exactly: q is u / D already
    for u, D in ((6.0, 3.0), (-1.5, 0.5), (1.0, 1024.0), (7.0, -7.0)):
        assert div_by_recip(u, D) == u / D


def test_select_is_what_keeps_minus_zero():
    # without the r == 0 select, fma(+0, y, -0) = +0 would replace -0 / D = -0 for D > 0
    u, D = -0.0, 3.0
    y = 1.0 / D
    q = u * y
    r = fma(-D, q, u)
    assert r == 0.0 and bits(fma(r, y, q)) != bits(u / D)
    assert bits(div_by_recip(u, D)) == bits(u / D)


@pytest.mark.parametrize("seed", [21, 22])
def test_window_edges_and_extreme_numerators(seed):
    """Quotients near the window's bounds and numerators far outside the normal range give
    IEEE's quotient for every divisor of the pivot range."""
    rng = random.Random(seed)
    for _ in range(4000):
        D = math.ldexp(1.0 + rng.random(), rng.randrange(-40, 1000)) * rng.choice((1, -1))
        eq = rng.choice((-900, 1000, -1074, -1030, 1023)) + rng.randrange(-40, 41)
        u = math.ldexp(1.0 + rng.random(), max(-1074, min(1023, eq + math.frexp(D)[1] - 1))) * rng.choice((1, -1))
        if math.isinf(u) or math.isinf(u / D):
            continue
        assert bits(div_by_recip(u, D)) == bits(u / D), (u, D)
    for D in (2.0 ** -40, -(2.0 ** 1000)):
        for u in (5e-324, -1e-310, 1.5, 1e300):
            assert bits(div_by_recip(u, D)) == bits(u / D), (u, D)


def test_correction_step_alone_fails_outside_the_window():
    """Why the window exists: with a numerator near or below the subnormal range the residual
    u - D q is not representable, and the correction step alone misses IEEE's quotient (pairs
    found by a random search, divisors inside the pivot range); the windowed division gets
    each one right."""
    pairs = ((4.975557870573251e-308, 8.378700874162909e-07), (8.603338021107614e-308, 9.136363321040337e-10),
             (6.91176798910094e-310, 0.0005959288686505066), (5.281900801e-314, 3.3922226277560964e-10))
    for u, D in pairs:
        assert bits(correction_step(u, D)) != bits(u / D), (u, D)
        assert bits(div_by_recip(u, D)) == bits(u / D), (u, D)

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


def exp_within(x: float, lo: int, hi: int) -> bool:
    """lo <= unbiased exponent field of x <= hi (zeros and subnormals count as -1023)."""
    e = ((struct.unpack("<Q", struct.pack("<d", x))[0] >> 52) & 0x7FF) - 1023
    return lo <= e <= hi


def ieee_div(u: float, D: float) -> float:
    """RN(u / D) with IEEE 754's signed zeros and infinities (Python raises on D == 0)."""
    if D == 0.0:
        if u == 0.0 or math.isnan(u):
            return math.nan
        return math.copysign(math.inf, u) * math.copysign(1.0, D)
    return u / D


def div_by_recip(u: float, D: float) -> float:
    """The kernels' division: the correction step inside the exponent window, else IEEE."""
    if not exp_within(D, -1000, 1000):
        return ieee_div(u, D)
    y = 1.0 / D  # RN(1/D), as __drcp_rn
    q = u * y  # RN(u y)
    if u != 0.0 and not (exp_within(u, -960, 1020) and exp_within(q, -1000, 1000)):
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
        D = random_double(rng, 100)
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
def test_window_edges_and_extreme_pairs(seed):
    """Pairs near and beyond the window (subnormal quotients and numerators, divisors near
    the overflow range) give IEEE's quotient through the fallback."""
    rng = random.Random(seed)
    for _ in range(4000):
        eu = rng.choice((-960, 1020, -1074, -1030, 1023)) + rng.randrange(-40, 41)
        ed = rng.choice((-1000, 1000, 1023, -1060)) + rng.randrange(-40, 41)
        u = math.ldexp(1.0 + rng.random(), max(-1074, min(1023, eu))) * rng.choice((1, -1))
        D = math.ldexp(1.0 + rng.random(), max(-1074, min(1023, ed))) * rng.choice((1, -1))
        if D == 0.0 or math.isinf(u) or math.isinf(D):
            continue
        assert bits(div_by_recip(u, D)) == bits(u / D), (u, D)


def test_correction_step_alone_fails_outside_the_window():
    """Why the window exists: with a subnormal numerator the residual u - D q is not
    representable, and the correction step alone misses IEEE's quotient (pairs found by a
    random search); the windowed division gets each one right."""
    pairs = ((8.83688982975e-313, 1.1789099603029609e-05), (1.350489187875e-312, 1.4922639623883187),
             (3.705522374004e-312, 7.22946908663457e-05), (1.4076e-320, 1.5708472293152395e-18))
    for u, D in pairs:
        assert bits(correction_step(u, D)) != bits(u / D), (u, D)
        assert bits(div_by_recip(u, D)) == bits(u / D), (u, D)

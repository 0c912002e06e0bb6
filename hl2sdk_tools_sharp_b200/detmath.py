"""Correctly rounded elementary functions for the host-side tables.

The reference computes a few of its lighting inputs with its own correctly
rounded math library (MapFormats/Numerics/DetMath.cs, DetMathF.cs), so
that every machine builds the same bits:

  * the 162 sky-ambient directions, DirectionalSampler.NextValue
    (MapTools/Rad/Light/DirectionalSampler.cs:96-121): DetMathF.Acos, Sin
    and Cos of float arguments;
  * the spotlight cone cosines and the sun's spread sine
    (Rad/Light/DirectLightBuilder.cs:385-386, 432): DetMath.CosToSingle and
    SinToSingle, the double result rounded again to float
    (DetMath.cs:151-187);
  * the light colours' gamma, RadLightFile.ParseIntensity
    (MapFormats/Text/RadLightFile.cs:383-396): DetMath.Pow in double;
  * LightNormals.FromProps (Rad/Light/LightNormals.cs:66-107);
  * the leaf ambient cone's tangent (Rad/Ambient/AmbientSampler.cs:142):
    DetMathF.Tan of a float.

These tables are made once per map on the host, so the functions here are
written for exactness, not speed: each value is evaluated in decimal at 60
significant digits or more (argument reduction by pi carried to as many
digits as the argument needs), converted exactly to a rational, and rounded
once to the target format, ties to even.  The reference's own tests pin the
same functions with a table of results computed at 3000 bits
(Tests/MapFormats/Numerics/DetMathGoldens.cs); tests/test_detmath_cpu.py
checks these functions against every row of it that they cover.
"""
from __future__ import annotations

import functools
import math
from decimal import Decimal, localcontext
from fractions import Fraction

import numpy as np

_PREC = 60


# ---------------------------------------------------------------- rounding

def _round_binary(q: Fraction, bits: int, emin: int) -> float:
    """q rounded to the nearest binary number with `bits` significant bits
    and exponents down to emin (subnormals below), ties to even."""
    if q == 0:
        return 0.0
    neg = q < 0
    q = -q if neg else q
    e = q.numerator.bit_length() - q.denominator.bit_length()
    if q < Fraction(2) ** e:
        e -= 1
    e = max(e, emin)
    shift = bits - 1 - e
    m = round(q * Fraction(2) ** shift)          # Fraction rounds ties to even
    v = math.ldexp(m, -shift)
    return -v if neg else v


def to_double(q) -> float:
    """The double nearest q (a Fraction or an exact Decimal)."""
    return _round_binary(Fraction(q), 53, -1022)


def to_single(q) -> np.float32:
    """The float nearest q."""
    return np.float32(_round_binary(Fraction(q), 24, -126))


# ---------------------------------------------------------------- kernels

@functools.lru_cache(maxsize=None)
def _pi(digits: int) -> Decimal:
    """pi to `digits` significant digits (Machin's formula)."""
    with localcontext() as c:
        c.prec = digits + 10

        def arctan_inv(n: int) -> Decimal:
            x = Decimal(1) / n
            x2 = x * x
            term, total, k = x, x, 1
            eps = Decimal(10) ** (-(digits + 8))
            while abs(term) > eps:
                term *= -x2
                k += 2
                total += term / k
            return total
        p = 16 * arctan_inv(5) - 4 * arctan_inv(239)
    with localcontext() as c:
        c.prec = digits
        return +p


def _digits_for(x: Decimal) -> int:
    return _PREC + max(0, x.adjusted()) + 10


def _sin_cos(x: Decimal) -> tuple[Decimal, Decimal]:
    """(sin x, cos x) to about _PREC digits, x exact."""
    prec = _digits_for(x)
    with localcontext() as c:
        c.prec = prec
        half_pi = _pi(prec) / 2
        k = int((x / half_pi).to_integral_value())
        r = x - k * half_pi
        r2 = r * r
        eps = Decimal(10) ** (-(prec - 2))
        s, term, n = r, r, 1
        while abs(term) > eps:
            term *= -r2 / ((n + 1) * (n + 2))
            n += 2
            s += term
        co, term, n = Decimal(1), Decimal(1), 0
        while abs(term) > eps:
            term *= -r2 / ((n + 1) * (n + 2))
            n += 2
            co += term
        q = k % 4
        return ((s, co), (co, -s), (-s, -co), (-co, s))[q]


def _atan(t: Decimal) -> Decimal:
    """atan t to about _PREC digits (t >= 0, exact)."""
    with localcontext() as c:
        c.prec = _PREC + 20
        if t > 1:
            return _pi(_PREC + 20) / 2 - _atan(1 / t)
        halvings = 0
        while t > Decimal("0.05"):
            t = t / (1 + (1 + t * t).sqrt())
            halvings += 1
        t2 = t * t
        term, total, k = t, t, 1
        eps = Decimal(10) ** (-(_PREC + 18))
        while abs(term) > eps:
            term *= -t2
            k += 2
            total += term / k
        return total * (2 ** halvings)


def _exact(x) -> Decimal:
    return Decimal(float(x))           # every binary float is an exact decimal


# ---------------------------------------------------------------- DetMath (double)

@functools.lru_cache(maxsize=1 << 16)
def sin_d(x: float) -> float:
    """DetMath.Sin: the double nearest sin x."""
    x = float(x)
    if x == 0.0 or not math.isfinite(x):
        return math.sin(x)
    return to_double(_sin_cos(_exact(x))[0])


@functools.lru_cache(maxsize=1 << 16)
def cos_d(x: float) -> float:
    """DetMath.Cos: the double nearest cos x."""
    x = float(x)
    if not math.isfinite(x):
        return math.cos(x)
    return to_double(_sin_cos(_exact(x))[1])


@functools.lru_cache(maxsize=1 << 16)
def pow_d(x: float, y: float) -> float:
    """DetMath.Pow for the arguments the lighting tables use (x >= 0):
    the double nearest x**y."""
    x, y = float(x), float(y)
    if y == 0.0 or x == 1.0:
        return 1.0
    if x < 0.0 or not (math.isfinite(x) and math.isfinite(y)):
        raise ValueError("pow_d covers finite x >= 0 only")
    if x == 0.0:
        return 0.0 if y > 0 else math.inf
    if y == int(y) and abs(y) <= 64:
        return to_double(Fraction(x) ** int(y))   # exact, so midpoints round right
    with localcontext() as c:
        c.prec = _PREC + 20
        v = (Decimal(y) * _exact(x).ln()).exp()
    return to_double(v)


def sin_to_single(x: float) -> np.float32:
    """DetMath.SinToSingle: sin x rounded to double, then to float."""
    return np.float32(sin_d(x))


def cos_to_single(x: float) -> np.float32:
    """DetMath.CosToSingle: cos x rounded to double, then to float."""
    return np.float32(cos_d(x))


# ---------------------------------------------------------------- DetMathF (float)

def sin_f(x) -> np.float32:
    """DetMathF.Sin: the float nearest sin x, x a float."""
    x = np.float32(x)
    if x == 0 or not np.isfinite(x):
        return np.float32(np.sin(x))
    return to_single(_sin_cos(_exact(x))[0])


def cos_f(x) -> np.float32:
    """DetMathF.Cos: the float nearest cos x, x a float."""
    x = np.float32(x)
    if not np.isfinite(x):
        return np.float32(np.cos(x))
    return to_single(_sin_cos(_exact(x))[1])


def tan_f(x) -> np.float32:
    """DetMathF.Tan: the float nearest tan x, x a float."""
    x = np.float32(x)
    if x == 0 or not np.isfinite(x):
        return np.float32(np.tan(x))
    s, c = _sin_cos(_exact(x))
    with localcontext() as ctx:
        ctx.prec = _PREC + 20
        return to_single(s / c)


def acos_f(x) -> np.float32:
    """DetMathF.Acos: the float nearest acos x, x a float in [-1, 1]."""
    x = np.float32(x)
    if not (-1 <= x <= 1):
        return np.float32(np.nan)
    if x == 1:
        return np.float32(0.0)
    d = _exact(x)
    with localcontext() as c:
        c.prec = _PREC + 20
        if x == -1:
            v = _pi(_PREC + 20)
        else:
            v = 2 * _atan(((1 - d) / (1 + d)).sqrt())
    return to_single(v)

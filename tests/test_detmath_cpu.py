"""The host-side correctly rounded functions (hl2sdk_tools_sharp_b200/detmath.py)
against the reference's DetMath golden table (DetMathGoldens.cs, computed
with mpmath at 3000 bits): every single-precision Acos, Sin, Cos and Tan row and
every double Sin, Cos and Pow row, bit for bit."""
import pathlib
import struct

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import detmath as DM

ROWS = pathlib.Path(__file__).resolve().parent / "golden" / "detmath-goldens-host.txt"


def _rows():
    out = []
    for line in ROWS.read_text().split("\n"):
        if line.strip():
            kind, fn, a, b, e = line.split()
            out.append((kind, fn, int(a, 16), int(b, 16), int(e, 16)))
    return out


def _f(bits):
    return np.uint32(bits).view(np.float32)


def _d(bits):
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


def _dbits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


FUNCS = {("F1", "Acos"): DM.acos_f, ("F1", "Sin"): DM.sin_f, ("F1", "Cos"): DM.cos_f, ("F1", "Tan"): DM.tan_f,
         ("D1", "Sin"): DM.sin_d, ("D1", "Cos"): DM.cos_d, ("D2", "Pow"): DM.pow_d}


@pytest.mark.parametrize("key", sorted(FUNCS))
def test_host_detmath_matches_the_golden_rows(key):
    rows = [r for r in _rows() if (r[0], r[1]) == key]
    assert len(rows) > 50
    fn = FUNCS[key]
    bad = []
    for kind, name, a, b, e in rows:
        if kind.startswith("F"):
            got = int(np.float32(fn(_f(a))).view(np.uint32))
            if np.isnan(_f(e)) and np.isnan(_f(got)):
                continue
        else:
            args = (_d(a),) if kind == "D1" else (_d(a), _d(b))
            if kind == "D2" and (_d(a) < 0 or not np.isfinite(_d(a)) or not np.isfinite(_d(b))):
                continue                    # outside the lighting tables' domain (x >= 0, finite)
            got = _dbits(fn(*args))
            if np.isnan(_d(e)) and np.isnan(_d(got)):
                continue
        if got != e:
            bad.append((name, hex(a), hex(b), hex(e), hex(got)))
    assert not bad, bad[:10]


def test_double_rounding_helpers_round_ties_to_even():
    from fractions import Fraction
    assert DM.to_single(Fraction(1) + Fraction(1, 2 ** 24)) == np.float32(1.0)
    assert DM.to_single(Fraction(1) + Fraction(3, 2 ** 24)) == np.float32(1.0) + np.float32(2.0 ** -22)
    assert DM.to_double(Fraction(1) + Fraction(1, 2 ** 53)) == 1.0

"""Form factors against the reference's known answers
(src/SourceSharp.Tests/MapTools/Rad/Bounce/FormFactorsTests.cs, the Correct
compliance cases), on the oracle (CPU) and on the device through the C ABI
(vrad_form_factor_diff / vrad_form_factor_poly, the functions the transfer
kernel calls); and device against oracle, bit for bit, on seeded cases."""
import math

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, tracer as T
from oracle import oracle as O

Z = np.zeros(3, np.float32)
UP = np.array([0, 0, 1], np.float32)
DOWN = np.array([0, 0, -1], np.float32)
A10 = np.array([0, 0, 10], np.float32)
SQUARE = np.array([[1, -1, 1], [1, 1, 1], [-1, 1, 1], [-1, -1, 1]], np.float32)
# The known-answer cases: (o1, n1, o2, n2) and what the reference asserts.
DIFF_CASES = [
    ((A10, DOWN, Z, UP), lambda f: f == pytest.approx(0.01, abs=5e-7)),   # facing: 1/r^2
    ((A10, UP, Z, UP), lambda f: f < 0),                                  # one facing away
    ((A10, UP, Z, DOWN), lambda f: f == pytest.approx(0.01, abs=5e-7)),   # both away: positive
]
POLY_CASES = [
    ((SQUARE, 4.0, Z, UP), lambda f: f * 4.0 / math.pi == pytest.approx(0.55412, abs=5e-5)),  # analytic
    ((SQUARE[::-1].copy(), 4.0, Z, UP), lambda f: f < 0),                                      # reversed
]


def test_oracle_form_factors_match_the_reference_cases():
    for args, ok in DIFF_CASES:
        assert ok(float(O.diff_to_diff(*args))), args
    for args, ok in POLY_CASES:
        assert ok(float(O.poly_to_diff(*args))), args


def _seeded(n=4000, seed=5):
    rng = np.random.default_rng(seed)
    diff = rng.normal(size=(n, 12)).astype(np.float32) * np.float32(50)
    for k in (3, 9):
        v = diff[:, k:k + 3]
        diff[:, k:k + 3] = (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)
    wind, cases = [], []
    for i in range(n // 4):
        k = int(rng.integers(3, 7))
        c = rng.normal(size=3) * 40
        ang = np.sort(rng.uniform(0, 2 * np.pi, k))
        r = rng.uniform(2, 30)
        pts = np.stack([c + r * np.array([np.cos(a), np.sin(a), 0]) for a in ang]).astype(np.float32)
        wind.append(pts)
        o = (c + rng.normal(size=3) * 20).astype(np.float32)
        nrm = rng.normal(size=3)
        nrm = (nrm / np.linalg.norm(nrm)).astype(np.float32)
        cases.append([np.float32(math.pi * r * r)] + list(o) + list(nrm))
    return diff, wind, np.array(cases, np.float32)


@pytest.mark.gpu
def test_device_form_factors_match_the_reference_cases_and_the_oracle():
    with T.CudaRayTracer(T.make_triangles(np.zeros((1, 9), np.float32) + np.arange(9, dtype=np.float32),
                                          np.zeros(1, np.int32))) as tr:
        got = L.form_factors_diff(tr, [np.concatenate(a) for a, _ in DIFF_CASES])
        for (args, ok), f in zip(DIFF_CASES, got):
            assert ok(float(f)), args
            assert f.view(np.uint32) == O.diff_to_diff(*args).view(np.uint32)
        got = L.form_factors_poly(tr, [a[0] for a, _ in POLY_CASES],
                                  [[a[1], *a[2], *a[3]] for a, _ in POLY_CASES])
        for (args, ok), f in zip(POLY_CASES, got):
            assert ok(float(f)), args
            assert f.view(np.uint32) == O.poly_to_diff(*args).view(np.uint32)
        diff, wind, cases = _seeded()
        got = L.form_factors_diff(tr, diff)
        want = np.array([O.diff_to_diff(d[0:3], d[3:6], d[6:9], d[9:12]) for d in diff], np.float32)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        got = L.form_factors_poly(tr, wind, cases)
        want = np.array([O.poly_to_diff(w, c[0], c[1:4], c[4:7]) for w, c in zip(wind, cases)], np.float32)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
